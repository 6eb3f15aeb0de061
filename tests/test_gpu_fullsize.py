"""Parity at the benchmark configurations' full sizes (not reduced cases).

Each test runs one benchmark configuration at its real size on the GPU and
compares it with the C oracle (itself pinned bit for bit to the reference's
own code by the golden fixtures):

* plain period sweep, 2^21 samples, nbins 128: the whole final fold and every
  score bit-exact, and the top-32 candidates;
* Taylor acceleration search, 2^22 samples, nbins 64, eta 2 (the benchmark
  line's workload): every score bit-exact, the S/N >= 7 candidates (indices
  and S/N bits) identical for FP32 and for BF16 fold storage, and the S/N
  error of both against the FP64 statement;
* jerk search through the pruning tree, 2^23 samples to 32 segments, one
  whole pruning run (31 levels, world tree 2^20, batches of 4096): FFA fold,
  per-level statistics and final tree bit-exact;
* Monte-Carlo cascade, 2^20 profiles x 64 bins, 8 stages: alive / kept
  profiles and every grid count bit-exact;
* a sample of the many-series workload (series of log-uniform length in
  2^18 .. 2^22, padded to powers of two): per-series candidates bit-exact.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import BENCH_WIDTHS
from oracle import lko

pytestmark = pytest.mark.gpu

W64 = np.array(BENCH_WIDTHS, dtype=np.uint64)


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def test_plain_sweep_2p21_nbins128_fold_and_scores(cuda):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA
    from loki_b200.synthetic import Pulsar, make_series

    nsamps, tsamp, nbins = 1 << 21, 64e-6, 128
    ts_e, ts_v = make_series(nsamps, tsamp, 42, [Pulsar(f0=1.0 / 0.0473, duty=0.05, snr=15.0)], nbins,
                             BENCH_WIDTHS)
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, 1.0, np.array([[5.0, 50.0]]), use_fourier=False,
                             score_widths=BENCH_WIDTHS)
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, 1.0, [[5.0, 50.0]]))
    ffa = FFACUDA(cfg)
    want_fold = lko.ffa(op, ts_e, ts_v)
    got_fold = ffa.execute(ts_e, ts_v)
    assert got_fold.size == want_fold.size == 773_095 * 2 * nbins
    np.testing.assert_array_equal(_bits(got_fold), _bits(want_fold))
    want = lko.snr_boxcar_3d(want_fold, W64, nbins).ravel()
    del want_fold, got_fold
    got = ffa.scores(ts_e, ts_v)
    np.testing.assert_array_equal(_bits(got), _bits(want))
    # top-32 candidates by S/N (ties: lower flat index first)
    top_w = np.lexsort((np.arange(want.size), -want))[:32]
    top_g = np.lexsort((np.arange(got.size), -got))[:32]
    np.testing.assert_array_equal(top_g, top_w)
    # the injected pulsar (fold S/N ~ 15) is the strongest detection
    assert want[top_w[0]] > 12.0


@pytest.mark.parametrize("storage", ["fp32", "bf16"])
def test_accel_search_2p22_candidates(cuda, storage):
    """The benchmark line's workload: candidates identical to the oracle's
    (indices and S/N bits) for both fold storages; FP32 scores bit-exact."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA
    from loki_b200.synthetic import taylor_accel_workload

    ts_e, ts_v, p, _ = taylor_accel_workload(seed=7)
    cfg = PulsarSearchConfig(p["nsamps"], p["tsamp"], p["nbins"], p["eta"], np.array(p["param_limits"]),
                             use_fourier=False, score_widths=p["score_widths"])
    op = lko.plan_create(lko.make_cfg(p["nsamps"], p["tsamp"], p["nbins"], p["eta"], p["param_limits"]))
    want = lko.snr_boxcar_3d(lko.ffa(op, ts_e, ts_v), W64, p["nbins"]).ravel()
    assert want.size == 1_932_740 * 8
    w_idx = np.flatnonzero(want >= 7.0)
    ffa = FFACUDA(cfg, fold_storage=storage)
    idx, snr, total = ffa.search(ts_e, ts_v, snr_min=7.0, max_cands=1 << 20)
    assert total == w_idx.size == 3729
    np.testing.assert_array_equal(idx.astype(np.int64), w_idx)
    np.testing.assert_array_equal(_bits(snr), _bits(want[w_idx]))
    if storage == "fp32":
        np.testing.assert_array_equal(_bits(ffa.scores(ts_e, ts_v)), _bits(want))


def test_accel_search_2p22_error_statement(cuda):
    """S/N error against the FP64 statement on the benchmark workload: FP32
    scores within 1e-4 everywhere; the BF16 search's candidates (exactly
    rescored) within 1e-4; BF16-stored scores' error recorded."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA
    from loki_b200.synthetic import taylor_accel_workload

    ts_e, ts_v, p, _ = taylor_accel_workload(seed=7)
    cfg = PulsarSearchConfig(p["nsamps"], p["tsamp"], p["nbins"], p["eta"], np.array(p["param_limits"]),
                             use_fourier=False, score_widths=p["score_widths"])
    op = lko.plan_create(lko.make_cfg(p["nsamps"], p["tsamp"], p["nbins"], p["eta"], p["param_limits"]))
    s64 = lko.ffa_scores64(op, ts_e, ts_v, W64).ravel()
    s32 = FFACUDA(cfg).scores(ts_e, ts_v).astype(np.float64)
    mixed = FFACUDA(cfg, fold_storage="bf16")
    s16 = mixed.scores(ts_e, ts_v).astype(np.float64)
    idx, snr, total = mixed.search(ts_e, ts_v, snr_min=7.0, max_cands=1 << 20)
    e32 = float(np.max(np.abs(s32 - s64)))
    ec = float(np.max(np.abs(snr.astype(np.float64) - s64[idx]))) if total else 0.0
    e16 = float(np.max(np.abs(s16 - s64)))
    print("ERRSTAT_2P22", {"fp32_max": e32, "bf16_candidates_max": ec, "bf16_all_cells_max": e16,
                           "bf16_all_cells_rms": float(np.sqrt(np.mean((s16 - s64) ** 2))), "candidates": total})
    assert e32 < 1e-4
    assert ec < 1e-4
    assert e16 < 0.1


def test_jerk_prune_2p23_whole_run(cuda):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA
    from loki_b200.prune import PruneCUDA, branching_pattern
    from loki_b200.synthetic import jerk_prune_workload

    ts_e, ts_v, p, thr, _ = jerk_prune_workload()
    cfg = PulsarSearchConfig(p["nsamps"], p["tsamp"], p["nbins"], p["eta"], np.array(p["param_limits"]),
                             use_fourier=False, bseg_ffa=p["bseg_ffa"])
    op = lko.plan_create(lko.make_cfg(p["nsamps"], p["tsamp"], p["nbins"], p["eta"], p["param_limits"],
                                      bseg_ffa=p["bseg_ffa"]))
    want_fold = lko.ffa(op, ts_e, ts_v)
    fold = FFACUDA(cfg).execute(ts_e, ts_v)
    np.testing.assert_array_equal(_bits(fold), _bits(want_fold))
    nseg = int(op.nsegments[-1])
    assert nseg == 32
    ms, bs = 1 << 20, 4096
    bm = max(int(np.ceil(branching_pattern(cfg, 0, False).max() * 2)), 32)
    want = lko.prune_run(op, want_fold, thr, nseg // 2, ms, bs, bm, nseg - 1)
    pr = PruneCUDA(cfg, max_sugg=ms, batch_size=bs)
    stats = pr.run(fold, nseg // 2, thr)
    for k in ("level", "seg_idx", "n_branches", "n_leaves", "n_leaves_phy", "n_leaves_surv", "threshold",
              "score_min", "score_max"):
        np.testing.assert_array_equal(stats[k], want[0][k])
    leaves, folds, scores = pr.tree()
    np.testing.assert_array_equal(leaves.view(np.uint64), want[1].view(np.uint64))
    np.testing.assert_array_equal(_bits(folds), _bits(want[2]))
    np.testing.assert_array_equal(_bits(scores), _bits(want[3]))
    assert int(stats["n_leaves"].sum()) > 100_000


def test_mc_cascade_2p20_profiles_8_stages(cuda):
    from loki_b200.synthetic import mc_cascade_workload
    from loki_b200.thresholds import mc_cascade

    folds0, signal, cls, noises, thresholds, grids = mc_cascade_workload()
    assert folds0.shape == (1 << 20, 64) and len(noises) == 8
    got = mc_cascade(folds0, signal, noises, cls, W64.astype(np.uint32), thresholds, grids)
    fin, rows, var = folds0, np.arange(folds0.shape[0], dtype=np.uint32), 1.0
    assert len(got) == 8
    for s, g in enumerate(got):
        f, ids, counts, _ = lko.mc_stage(fin, noises[s], signal, var, var, W64, thresholds[s], grids[s],
                                         signal_scale=float(2 ** s), rowmap=rows, cls=cls)
        ng = len(grids[s])
        assert (g["alive"], g["kept"]) == (rows.size, ids.size)
        np.testing.assert_array_equal(g["counts"].astype(np.uint64), counts[:ng])
        np.testing.assert_array_equal(g["counts_flagged"].astype(np.uint64), counts[ng:])
        fin, rows, var = f, ids, 2 * var
    assert 0 < got[-1]["kept"] < got[0]["alive"]


def test_many_series_sample_uneven_lengths(cuda):
    """Eight series of the many-series workload's shape (log-uniform lengths
    in 2^18 .. 2^22, one in eight with a pulsar, nbins 128, f 2-50 Hz), padded
    to powers of two and batched by length: per-series candidates exact."""
    from loki_b200.batched import MultiSeriesSearch
    from loki_b200.synthetic import multi_series_workload

    data, p = multi_series_workload(nseries=8, seed=3)
    thr = 6.0
    res = MultiSeriesSearch(tsamp=p["tsamp"], nbins=p["nbins"], f_range=p["f_range"], widths=p["widths"],
                            snr_min=thr, max_batch=2).search(data)
    w64 = np.array(p["widths"], np.uint64)
    for (e, v), r in zip(data, res):
        L = 1 << int(np.ceil(np.log2(e.size)))
        ep = np.zeros(L, np.float32)
        vp = np.zeros(L, np.float32)
        ep[: e.size] = e
        vp[: e.size] = v
        plan = lko.plan_create(lko.make_cfg(L, p["tsamp"], p["nbins"], p["eta"], [list(p["f_range"])]))
        sc = lko.snr_boxcar_3d(lko.ffa(plan, ep, vp), w64, p["nbins"]).ravel()
        want = np.flatnonzero(sc >= thr)
        np.testing.assert_array_equal(r["idx"].astype(np.int64), want)
        np.testing.assert_array_equal(_bits(r["snr"]), _bits(sc[want]))
    assert max(e.size for e, _ in data) > 1 << 20
