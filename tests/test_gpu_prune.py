"""Pruning leaf step on the GPU (through the C ABI) against the C oracle and
the reference's own pruning runs: every step bit-exact (leaves are FP64 and
compared bit for bit; folds and scores are FP32 and compared bit for bit),
whole runs with identical per-level statistics and identical final trees,
including runs where the world tree overflows and the threshold is raised by
the overload rule."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import golden
from oracle import lko

pytestmark = pytest.mark.gpu

STAT_FIELDS = ("level", "seg_idx", "n_branches", "n_leaves", "n_leaves_phy", "n_leaves_surv",
               "threshold", "score_min", "score_max")

# nsamps, tsamp, nbins, eta, limits, bseg_ffa, seed, max_sugg, batch, thr_lo, thr_hi, ref_frac, conservative
CASES = {
    "accel_nb32_overload": (1 << 17, 1e-3, 32, 1.0, [[-20.0, 20.0], [5.0, 6.0]], 1 << 13, 1, 160, 16,
                            1.0, 3.0, 0.5, False),
    "accel_nb64_eta2": (1 << 19, 5e-4, 64, 2.0, [[-200.0, 200.0], [20.0, 25.0]], 1 << 14, 2, 4096, 64,
                        2.0, 5.0, 0.3, False),
    "accel_nb32_wrap": (1 << 17, 1e-3, 32, 1.0, [[-20.0, 20.0], [5.0, 7.0]], 1 << 13, 3, 301, 37,
                        0.5, 2.5, 1.0, True),
    "jerk_nb32_cons": (1 << 18, 1e-3, 32, 1.0, [[-0.2, 0.2], [-20.0, 20.0], [5.0, 6.0]], 1 << 14, 4, 400, 32,
                       1.0, 3.0, 0.2, True),
    "jerk_nb32_big": (1 << 19, 5e-4, 32, 1.0, [[-0.5, 0.5], [-30.0, 30.0], [20.0, 21.0]], 1 << 14, 5, 4133,
                      100, 2.0, 4.0, 0.7, False),
    # thousands of parents and children: multi-tile scans and compactions
    "accel_nb32_multitile": (1 << 20, 5e-4, 32, 1.0, [[-50.0, 50.0], [10.0, 14.0]], 1 << 15, 6, 5000, 1000,
                             1.0, 3.0, 0.5, False),
    "accel_nb32_many_batches": (1 << 20, 5e-4, 32, 1.0, [[-50.0, 50.0], [10.0, 14.0]], 1 << 15, 7, 1 << 15,
                                64, 1.0, 3.0, 0.25, False),
}


def _series(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n).astype(np.float32), (1.0 + 0.25 * rng.random(n)).astype(np.float32)


def _setup(name):
    from loki_b200.configs import PulsarSearchConfig

    ns, ts, nb, eta, lim, bf, seed, ms, bs, lo, hi, rf, cons = CASES[name]
    plan = lko.plan_create(lko.make_cfg(ns, ts, nb, eta, lim, bseg_ffa=bf))
    cfg = PulsarSearchConfig(ns, ts, nb, eta, np.array(lim), use_fourier=False, bseg_ffa=bf)
    e, v = _series(ns, seed)
    fold = lko.ffa(plan, e, v)
    nseg = int(plan.nsegments[-1])
    ref_seg = min(int(nseg * rf), nseg - 1)
    thr = np.linspace(lo, hi, nseg - 1).astype(np.float32)
    return plan, cfg, (e, v), fold, nseg, ref_seg, thr, ms, bs, cons


def _stats_matrix(stats):
    return np.stack([stats[k].astype(np.float64) for k in STAT_FIELDS], axis=1)


def _branch_max(cfg, cons):
    from loki_b200.prune import branching_pattern

    return max(int(np.ceil(branching_pattern(cfg, 0, cons).max() * 2)), 32)


@pytest.mark.parametrize("name", sorted(CASES))
def test_prune_run_bit_exact(cuda, name):
    from loki_b200.prune import PruneCUDA

    plan, cfg, _, fold, nseg, ref_seg, thr, ms, bs, cons = _setup(name)
    bm = _branch_max(cfg, cons)
    want = lko.prune_run(plan, fold, thr, ref_seg, ms, bs, bm, nseg - 1, conservative=cons)
    pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs, branch_max=None, use_conservative_tile=cons)
    stats = pr.run(fold, ref_seg, thr)
    np.testing.assert_array_equal(_stats_matrix(stats), _stats_matrix(want[0]))
    leaves, folds, scores = pr.tree()
    np.testing.assert_array_equal(leaves, want[1])
    np.testing.assert_array_equal(folds, want[2])
    np.testing.assert_array_equal(scores, want[3])
    # a second run on the same executor starts from a clean tree
    stats2 = pr.run(fold, ref_seg, thr)
    np.testing.assert_array_equal(_stats_matrix(stats2), _stats_matrix(want[0]))


@pytest.mark.parametrize("name", ["accel_nb32_overload", "accel_nb32_wrap", "accel_nb32_many_batches",
                                  "jerk_nb32_big"])
def test_prune_tail_matches_level_by_level(cuda, name):
    """The persistent tail (small trees in one cooperative launch, batch
    replay on the device; hands large levels back) gives exactly the
    level-by-level run: statistics, leaves, folds, scores."""
    from loki_b200.prune import PruneCUDA

    plan, cfg, _, fold, nseg, ref_seg, thr, ms, bs, cons = _setup(name)
    runs = []
    for tail in (False, True):
        pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs, branch_max=None, use_conservative_tile=cons)
        pr.set_persistent_tail(tail)
        stats = pr.run(fold, ref_seg, thr)
        runs.append((_stats_matrix(stats), pr.tree()))
    (s0, t0), (s1, t1) = runs
    np.testing.assert_array_equal(s1, s0)
    for a, b in zip(t0, t1):
        np.testing.assert_array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("name", ["accel_nb32_overload", "accel_nb32_many_batches", "jerk_nb32_big",
                                  "accel_nb32_wrap"])
def test_prune_run_many_matches_single_runs(cuda, name):
    """Several runs with their tails in one cooperative launch (run_many) give
    each run's own result; the many-batches case hands levels back."""
    from loki_b200.prune import PruneCUDA

    plan, cfg, _, fold, nseg, _, thr, ms, bs, cons = _setup(name)
    segs = sorted({0, nseg // 3, nseg // 2, nseg - 1})
    kw = dict(max_sugg=ms, batch_size=bs, branch_max=None, use_conservative_tile=cons)
    many = [PruneCUDA(cfg, **kw) for _ in segs]
    got = PruneCUDA.run_many(many, fold, segs, thr)
    for pr, rs, st in zip(many, segs, got):
        one = PruneCUDA(cfg, **kw)
        want = one.run(fold, rs, thr)
        np.testing.assert_array_equal(_stats_matrix(st), _stats_matrix(want))
        for a, b in zip(pr.tree(), one.tree()):
            np.testing.assert_array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("name", ["prune_accel_nb16.npz", "prune_jerk_nb16.npz"])
def test_prune_reference_golden_fixtures(cuda, name):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.prune import PruneCUDA

    g = golden(name)
    cfg = PulsarSearchConfig(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                             g["param_limits"], use_fourier=False, bseg_ffa=int(g["bseg_ffa"]))
    pr = PruneCUDA(cfg, max_sugg=int(g["max_sugg"]), batch_size=int(g["batch_size"]),
                   branch_max=int(g["branch_max"]), use_conservative_tile=bool(g["conservative"]))
    stats = pr.run(g["ffa_fold"], int(g["ref_seg"]), g["thresholds"])
    np.testing.assert_array_equal(_stats_matrix(stats), g["stats"])
    leaves, folds, scores = pr.tree()
    np.testing.assert_array_equal(leaves, g["leaves"])
    np.testing.assert_array_equal(folds, g["folds"])
    np.testing.assert_array_equal(scores, g["scores"])


def test_ep_multipass_end_to_end(cuda):
    """FFA on the GPU, then one pruning run per reference segment."""
    from loki_b200.prune import EPMultiPassCUDA, determine_ref_segs

    plan, cfg, (e, v), fold, nseg, _, thr, ms, bs, cons = _setup("accel_nb32_overload")
    ep = EPMultiPassCUDA(cfg, thr, n_runs=3, max_sugg=ms, batch_size=bs)
    res = ep.execute(e, v)
    bm = _branch_max(cfg, False)
    assert sorted(res) == sorted(determine_ref_segs(nseg, 3))
    for rs, r in res.items():
        want = lko.prune_run(plan, fold, thr, rs, ms, bs, bm, nseg - 1)
        np.testing.assert_array_equal(_stats_matrix(r["stats"]), _stats_matrix(want[0]))
        # survivors ascended and reported as PruneImpl::run ends
        lv, fo, sc, ep = lko.prune_finalize(plan, fold, rs, want[0].size - 1, *want[1:])
        np.testing.assert_array_equal(r["leaves"], lv)
        np.testing.assert_array_equal(r["folds"], fo)
        np.testing.assert_array_equal(r["scores"], sc)
        np.testing.assert_array_equal(r["scores_ep"], ep)
        assert r["snail_scheme"][0] == rs


def test_ep_multipass_concurrent_runs_identical(cuda, tmp_path):
    """Reference segments run on 3 executors at once (own streams and host
    threads) give exactly the sequential results, and the .npz holds one run
    group per segment."""
    from loki_b200.prune import EPMultiPassCUDA

    plan, cfg, (e, v), fold, nseg, _, thr, ms, bs, cons = _setup("accel_nb32_many_batches")
    seq = EPMultiPassCUDA(cfg, thr, n_runs=5, max_sugg=ms, batch_size=bs, n_workers=1).execute(e, v)
    par = EPMultiPassCUDA(cfg, thr, n_runs=5, max_sugg=ms, batch_size=bs, n_workers=3).execute(
        e, v, outdir=str(tmp_path), file_prefix="t")
    thr_par = EPMultiPassCUDA(cfg, thr, n_runs=5, max_sugg=ms, batch_size=bs, n_workers=3,
                              batched=False).execute(e, v)
    assert sorted(seq) == sorted(par) == sorted(thr_par) and len(seq) == 5
    for other in (par, thr_par):
        for rs in seq:
            for k in ("leaves", "folds", "scores", "scores_ep"):
                np.testing.assert_array_equal(other[rs][k].view(np.uint8), seq[rs][k].view(np.uint8))
            np.testing.assert_array_equal(_stats_matrix(other[rs]["stats"]), _stats_matrix(seq[rs]["stats"]))
    z = np.load(tmp_path / f"t_pruning_nstages_{nseg}_results.npz")
    for rs in seq:
        np.testing.assert_array_equal(z[f"{rs:03d}_00/param_sets"], seq[rs]["leaves"])
        np.testing.assert_array_equal(z[f"{rs:03d}_00/scores_ep"], seq[rs]["scores_ep"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_prune_finalize_bit_exact(cuda, name):
    """Ascend + report (the end of PruneImpl::run) after full and partial runs."""
    from loki_b200.prune import PruneCUDA

    plan, cfg, _, fold, nseg, ref_seg, thr, ms, bs, cons = _setup(name)
    bm = _branch_max(cfg, cons)
    pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs, branch_max=None, use_conservative_tile=cons)
    for n_iters in (nseg - 1, max(1, (nseg - 1) // 3)):
        want = lko.prune_run(plan, fold, thr, ref_seg, ms, bs, bm, n_iters, conservative=cons)
        lv, fo, sc, ep = lko.prune_finalize(plan, fold, ref_seg, want[0].size - 1, *want[1:])
        pr.run(fold, ref_seg, thr, n_iters=n_iters)
        pr.finalize(fold)
        leaves, folds, scores = pr.tree()
        np.testing.assert_array_equal(leaves.view(np.uint64), lv.view(np.uint64))
        np.testing.assert_array_equal(folds.view(np.uint32), fo.view(np.uint32))
        np.testing.assert_array_equal(scores.view(np.uint32), sc.view(np.uint32))
        np.testing.assert_array_equal(pr.scores_ep().view(np.uint32), ep.view(np.uint32))


@pytest.mark.parametrize("name", ["prune_accel_nb16.npz", "prune_jerk_nb16.npz", "prune_cheby_accel_nb16.npz",
                                  "prune_cheby_jerk_nb16.npz"])
@pytest.mark.parametrize("tag", ["final", "half"])
def test_prune_finalize_reference_golden_fixtures(cuda, name, tag):
    from loki_b200 import _capi as C
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.prune import PruneCUDA

    g = golden(name)
    cfg = PulsarSearchConfig(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                             g["param_limits"], use_fourier=False, bseg_ffa=int(g["bseg_ffa"]))
    pr = PruneCUDA(cfg, max_sugg=int(g["max_sugg"]), batch_size=int(g["batch_size"]),
                   branch_max=int(g["branch_max"]), use_conservative_tile=bool(g["conservative"]),
                   poly_basis=str(g["basis"]))
    nseg = g["thresholds"].size + 1
    n_iters = nseg - 1 if tag == "final" else (nseg - 1) // 2
    with pytest.raises(C.LokiError):
        pr.finalize(g["ffa_fold"])  # no run yet
    stats = pr.run(g["ffa_fold"], int(g["ref_seg"]), g["thresholds"], n_iters=n_iters)
    assert stats.size - 1 == int(g[f"{tag}_levels"])
    pr.finalize(g["ffa_fold"])
    with pytest.raises(C.LokiError):
        pr.finalize(g["ffa_fold"])  # once per run
    leaves, folds, scores = pr.tree()
    np.testing.assert_array_equal(leaves.view(np.uint64), g[f"{tag}_leaves"].view(np.uint64))
    np.testing.assert_array_equal(folds.view(np.uint32), g[f"{tag}_folds"].view(np.uint32))
    np.testing.assert_array_equal(scores.view(np.uint32), g[f"{tag}_scores"].view(np.uint32))
    np.testing.assert_array_equal(pr.scores_ep().view(np.uint32), g[f"{tag}_scores_ep"].view(np.uint32))


# ---- single steps ---------------------------------------------------------------

def _dev(t, a, dtype=None):
    return t.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype))).cuda()


def _stream(t):
    return t.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("name", ["accel_nb32_overload", "jerk_nb32_cons"])
def test_steps_bit_exact(cuda, name):
    from loki_b200 import _capi as C

    t = cuda
    L = C.lib()
    plan, cfg, _, fold, nseg, ref_seg, thr, ms, bs, cons = _setup(name)
    np_ = plan.nparams
    nb = plan.nbins
    nc = int(plan.ncoords[-1])
    h = cfg._plan_handle
    s = _stream(t)

    # seed
    seed_want = lko.taylor_seed(plan)
    d_seed = t.empty((nc, np_ + 2, 2), dtype=t.float64, device="cuda")
    C.check(L.lk_taylor_seed(h, d_seed.data_ptr(), s))
    np.testing.assert_array_equal(d_seed.cpu().numpy(), seed_want)

    # branch at levels 1..3 of the middle-out order (branching happens at some)
    tseg = float(cfg.tseg_ffa)
    leaves = seed_want
    bm = _branch_max(cfg, cons)
    for level in (1, 2, 3):
        _, coord, cur, segc = lko.middle_out(nseg, ref_seg, tseg, level)
        want_l, want_o = lko.taylor_branch(leaves, np_, cur, nb, float(cfg.eta), bm)
        d_in = _dev(t, leaves)
        cap = want_l.shape[0] + 5
        d_out = t.empty((cap, np_ + 2, 2), dtype=t.float64, device="cuda")
        d_org = t.empty(cap, dtype=t.int32, device="cuda")
        n = ctypes.c_uint64()
        C.check(L.lk_taylor_branch(h, d_in.data_ptr(), leaves.shape[0], cur[1], bm, d_out.data_ptr(),
                                   d_org.data_ptr(), cap, ctypes.byref(n), s))
        assert n.value == want_l.shape[0]
        np.testing.assert_array_equal(d_out[: n.value].cpu().numpy(), want_l)
        np.testing.assert_array_equal(d_org[: n.value].cpu().numpy().astype(np.uint64), want_o)

        # resolve against the segment of this level
        _, c_init, _, _ = lko.middle_out(nseg, ref_seg, tseg, 0)
        coords = np.array([*segc, *cur, *c_init], np.float64)
        pidx_w, ph_w = lko.taylor_resolve(plan, want_l, segc, cur, c_init)
        d_pidx = t.empty(n.value, dtype=t.int32, device="cuda")
        d_ph = t.empty(n.value, dtype=t.float32, device="cuda")
        C.check(L.lk_taylor_resolve(h, d_out.data_ptr(), n.value, coords.ctypes.data, d_pidx.data_ptr(),
                                    d_ph.data_ptr(), s))
        np.testing.assert_array_equal(d_pidx.cpu().numpy().astype(np.uint64), pidx_w)
        np.testing.assert_array_equal(d_ph.cpu().numpy(), ph_w)

        # transform every other leaf, both tile modes
        idx = np.arange(0, n.value, 2, dtype=np.uint64)
        for c in (False, True):
            tw = lko.taylor_transform(want_l, idx, np_, coord, cur, c)
            d_t = _dev(t, want_l)
            d_idx = _dev(t, idx, np.int32)
            C.check(L.lk_taylor_transform(h, d_t.data_ptr(), n.value, d_idx.data_ptr(), idx.size, coord[0],
                                          cur[0], int(c), s))
            np.testing.assert_array_equal(d_t.cpu().numpy(), tw)
        leaves = lko.taylor_transform(want_l, np.arange(n.value, dtype=np.uint64), np_, coord, cur, cons)


def test_shift_add_and_score_filter_bit_exact(cuda):
    from loki_b200 import _capi as C

    t = cuda
    L = C.lib()
    rng = np.random.default_rng(11)
    nb, cap, nffa, n = 48, 37, 23, 500
    tree = np.empty((cap, 2, nb), np.float32)
    tree[:, 0] = rng.standard_normal((cap, nb)) * 5
    tree[:, 1] = 20 + rng.random((cap, nb)) * 5
    ffa = np.empty((nffa, 2, nb), np.float32)
    ffa[:, 0] = rng.standard_normal((nffa, nb)) * 5
    ffa[:, 1] = 20 + rng.random((nffa, nb)) * 5
    it = rng.integers(0, 20, n).astype(np.uint64)
    iff = rng.integers(0, nffa, n).astype(np.uint64)
    ph = (rng.random(n) * nb).astype(np.float32)
    ph[:5] = [0.0, nb - 0.5, nb - 0.50001, 0.49999, 0.5]
    pstart = 30
    want = lko.shift_add_batch(tree, it, ffa, iff, ph, nb, pstart, cap)
    # keep every device buffer referenced for as long as the library uses it
    d_tree, d_it, d_ffa, d_iff, d_ph = (_dev(t, tree), _dev(t, it, np.int32), _dev(t, ffa),
                                        _dev(t, iff, np.int32), _dev(t, ph))
    d_out = t.empty((n, 2, nb), dtype=t.float32, device="cuda")
    s = _stream(t)
    C.check(L.lk_shift_add_batch(d_tree.data_ptr(), d_it.data_ptr(), d_ffa.data_ptr(), nffa, d_iff.data_ptr(),
                                 d_ph.data_ptr(), d_out.data_ptr(), nb, n, pstart, cap, s))
    np.testing.assert_array_equal(d_out.cpu().numpy(), want)
    # an FFA row beyond n_ffa is rejected by the kernel's bounds check
    rc = L.lk_shift_add_batch(d_tree.data_ptr(), d_it.data_ptr(), d_ffa.data_ptr(), nffa - 1, d_iff.data_ptr(),
                              d_ph.data_ptr(), d_out.data_ptr(), nb, n, pstart, cap, s)
    assert rc == C.LK_ERR_INVALID_ARG

    widths = np.array([1, 2, 3, 5, 8, 13], np.uint32)
    sc_w, idx_w = lko.score_filter(want, nb, widths.astype(np.uint64), 4.0)
    d_out = _dev(t, want)
    d_sc = t.empty(n, dtype=t.float32, device="cuda")
    d_idx = t.empty(n, dtype=t.int32, device="cuda")
    d_cnt = t.zeros(1, dtype=t.int64, device="cuda")
    C.check(L.lk_score_filter(d_out.data_ptr(), n, nb, widths.ctypes.data, widths.size, 4.0, d_sc.data_ptr(),
                              d_idx.data_ptr(), d_cnt.data_ptr(), s))
    np.testing.assert_array_equal(d_sc.cpu().numpy(), sc_w)
    k = int(d_cnt.item())
    assert k == idx_w.size and 0 < k < n
    np.testing.assert_array_equal(d_idx[:k].cpu().numpy().astype(np.uint64), idx_w)


def test_prune_errors_are_loud(cuda):
    from loki_b200 import LokiError
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.prune import PruneCUDA

    plan, cfg, _, fold, nseg, ref_seg, thr, ms, bs, cons = _setup("accel_nb32_overload")
    with pytest.raises(LokiError, match="Suggestions too large"):
        PruneCUDA(cfg, max_sugg=int(plan.ncoords[-1]) - 1, batch_size=bs)
    pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs, branch_max=1)
    with pytest.raises(LokiError, match="branch_max"):
        pr.run(fold, ref_seg, thr)
    pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs)
    with pytest.raises(LokiError, match="ref_idx"):
        pr.run(fold, nseg, thr)
    with pytest.raises(LokiError, match="threshold scheme"):
        pr.run(fold, ref_seg, thr[:2], n_iters=5)
    freq_cfg = PulsarSearchConfig(1 << 15, 1e-3, 32, 1.0, np.array([[5.0, 6.0]]), use_fourier=False)
    with pytest.raises(NotImplementedError):
        PruneCUDA(freq_cfg)
