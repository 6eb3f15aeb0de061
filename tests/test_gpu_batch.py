"""Batched FFA executor on the GPU: every series of a batch gets exactly its
single-series result (the batch is one launch per level), search indices are
flat over the batch, and a CUDA-graph capture of a batch step replays to the
same result; the multi-series driver pads, groups and matches the oracle."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import series
from oracle import lko

pytestmark = pytest.mark.gpu


def _cfg(nsamps, nbins=32, lims=((-300.0, 300.0), (5.0, 8.0)), tsamp=1e-3, widths=(1, 2, 3, 4, 6)):
    from loki_b200.configs import PulsarSearchConfig

    return PulsarSearchConfig(nsamps, tsamp, nbins, 1.0, np.array(lims), use_fourier=False,
                              score_widths=list(widths))


@pytest.mark.parametrize("nbins,lims", [(32, ((-300.0, 300.0), (5.0, 8.0))), (128, ((20.0, 40.0),))])
def test_batch_matches_single_series(cuda, nbins, lims):
    from loki_b200.ffa import FFACUDA

    t = cuda
    n, nb = 1 << 17, 3
    cfg = _cfg(n, nbins, lims, tsamp=1e-3 if len(lims) == 2 else 64e-6)
    single = FFACUDA(cfg)
    batched = FFACUDA(cfg, max_batch=4)
    es, vs = zip(*(series(n, 40 + k) for k in range(nb)))
    e = t.from_numpy(np.stack(es)).cuda()
    v = t.from_numpy(np.stack(vs)).cuda()
    got = batched.scores_batch(e, v).cpu().numpy()
    for k in range(nb):
        want = single.scores(es[k], vs[k])
        np.testing.assert_array_equal(got[k].view(np.uint32), want.view(np.uint32))
    # search indices flat over [series][coord][width]
    thr = float(np.quantile(got, 0.999))
    idx, snr, total = batched.search_batch(e, v, snr_min=thr)
    flat = got.ravel()
    want_idx = np.flatnonzero(flat >= thr)
    assert total == want_idx.size
    np.testing.assert_array_equal(idx, want_idx.astype(np.uint32))
    np.testing.assert_array_equal(snr, flat[want_idx])


def test_batch_graph_replay(cuda):
    from loki_b200.ffa import FFACUDA

    t = cuda
    n, nb = 1 << 16, 2
    cfg = _cfg(n)
    ffa = FFACUDA(cfg, max_batch=nb)
    e = t.empty((nb, n), dtype=t.float32, device="cuda")
    v = t.empty((nb, n), dtype=t.float32, device="cuda")
    idx = t.empty(1 << 16, dtype=t.int32, device="cuda")
    snr = t.empty(1 << 16, dtype=t.float32, device="cuda")
    cnt = t.zeros(1, dtype=t.int64, device="cuda")
    es, vs = zip(*(series(n, 60 + k) for k in range(nb)))
    e.copy_(t.from_numpy(np.stack(es)))
    v.copy_(t.from_numpy(np.stack(vs)))
    ffa.search_batch(e, v, 3.0, idx, snr, cnt)  # warm-up: allocations happen here
    t.cuda.synchronize()
    eager = (idx[: int(cnt.item())].clone(), snr[: int(cnt.item())].clone())
    g = t.cuda.CUDAGraph()
    with t.cuda.graph(g):
        ffa.search_batch(e, v, 3.0, idx, snr, cnt)
    for k in range(2):
        es2, vs2 = zip(*(series(n, 70 + 10 * k + j) for j in range(nb)))
        e.copy_(t.from_numpy(np.stack(es2)))
        v.copy_(t.from_numpy(np.stack(vs2)))
        g.replay()
        t.cuda.synchronize()
        got = (idx[: int(cnt.item())].cpu().numpy(), snr[: int(cnt.item())].cpu().numpy())
        ffa.search_batch(e, v, 3.0, idx, snr, cnt)
        t.cuda.synchronize()
        np.testing.assert_array_equal(got[0], idx[: int(cnt.item())].cpu().numpy())
        np.testing.assert_array_equal(got[1], snr[: int(cnt.item())].cpu().numpy())
    assert eager[0].numel() > 0


def test_multi_series_driver_matches_oracle(cuda):
    from loki_b200.batched import MultiSeriesSearch

    lengths = [3000, 5000, 9000, 16384, 20000, 70000]
    rng = np.random.default_rng(5)
    data = [(rng.standard_normal(L).astype(np.float32), np.ones(L, np.float32)) for L in lengths]
    widths = [1, 2, 3, 4, 6, 8]
    ms = MultiSeriesSearch(tsamp=1e-3, nbins=32, f_range=(5.0, 9.0), widths=widths, snr_min=3.5, max_batch=2)
    res = ms.search(data)
    for (e, v), r in zip(data, res):
        L = 1 << int(np.ceil(np.log2(e.size)))
        ep = np.zeros(L, np.float32)
        vp = np.zeros(L, np.float32)
        ep[: e.size] = e
        vp[: e.size] = v
        plan = lko.plan_create(lko.make_cfg(L, 1e-3, 32, 1.0, [[5.0, 9.0]]))
        sc = lko.snr_boxcar_3d(lko.ffa(plan, ep, vp), np.array(widths, np.uint64), 32).ravel()
        want = np.flatnonzero(sc >= 3.5)
        np.testing.assert_array_equal(r["idx"], want.astype(np.uint32))
        np.testing.assert_array_equal(r["snr"], sc[want])


def test_search_pipeline_matches_search(cuda):
    """SearchPipeline (copies overlapped with searches) returns per series
    exactly what FFACUDA.search returns."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA
    from loki_b200.pipeline import SearchPipeline

    cfg = PulsarSearchConfig(2**18, 1e-3, 32, 1.0, np.array([[-300.0, 300.0], [5.0, 8.0]]), use_fourier=False,
                             score_widths=[1, 2, 3, 4])
    ffa = FFACUDA(cfg)
    data = [series(cfg.nsamps, 70 + k) for k in range(5)]
    s0 = ffa.scores(*data[0])
    thr = float(np.quantile(s0, 0.999))
    want = [ffa.search(e, v, snr_min=thr) for e, v in data]
    for n_exec in (1, 2, 3):
        got = list(SearchPipeline(ffa, thr, max_cands=1 << 16, n_exec=n_exec).run(data))
        assert len(got) == len(want)
        for (gi, gs, gn), (wi, ws, wn) in zip(got, want):
            assert gn == wn
            np.testing.assert_array_equal(gi, wi)
            np.testing.assert_array_equal(gs.view(np.uint32), ws.view(np.uint32))


@pytest.mark.parametrize("nbins,lims,storage", [(64, [[-200.0, 200.0], [5.0, 50.0]], "fp32"),
                                                (32, [[-300.0, 300.0], [5.0, 8.0]], "bf16"),
                                                (128, [[20.0, 60.0]], "fp32")])
def test_autotune_keeps_results(cuda, nbins, lims, storage):
    """The autotuner only changes launch shapes: scores stay bit-exact with
    the oracle and a BF16 search keeps the FP32 candidates."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA

    ns = 2**18
    cfg = PulsarSearchConfig(ns, 1e-3 if len(lims) == 2 and nbins == 32 else 64e-6, nbins, 1.0, np.array(lims),
                             use_fourier=False, score_widths=[1, 2, 3, 4])
    op = lko.plan_create(lko.make_cfg(ns, cfg.tsamp, nbins, 1.0, lims))
    e, v = series(ns, 91)
    ffa = FFACUDA(cfg, fold_storage=storage)
    t = ffa.autotune(e, v, reps=1)
    assert t["candidates"] > 3 and t["bf_rows"] in (1, 2) and t["bf_warps"] >= 1 and t["bf_stages"] >= 2
    assert ffa.tuning["bf_warps"] == t["bf_warps"]
    if storage == "fp32":
        want = lko.snr_boxcar_3d(lko.ffa(op, e, v), np.array([1, 2, 3, 4], np.uint64), nbins).ravel()
        got = ffa.scores(e, v)
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    else:
        plain = FFACUDA(cfg)
        thr = float(np.quantile(plain.scores(e, v), 0.999))
        a = plain.search(e, v, snr_min=thr)
        b = ffa.search(e, v, snr_min=thr)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    # a saved tuning applies to a fresh executor
    other = FFACUDA(cfg, fold_storage=storage)
    other.set_tuning(t)
    for k in ("bf_rows", "bf_warps", "bf_stages", "merge_rows_in_flight", "score_cells_per_block"):
        assert other.tuning[k] == t[k]


def test_autotune_multi_segment_plan(cuda):
    """A plan that stops at several segments (the pruning input) is tuned
    through its brute fold and merges; the fold stays bit-exact."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA

    ns, bseg = 2**18, 2**13
    lims = [[-20.0, 20.0], [5.0, 6.0]]
    cfg = PulsarSearchConfig(ns, 1e-3, 32, 1.0, np.array(lims), use_fourier=False, bseg_ffa=bseg)
    op = lko.plan_create(lko.make_cfg(ns, 1e-3, 32, 1.0, lims, bseg_ffa=bseg))
    assert op.nsegments[-1] > 1
    e, v = series(ns, 93)
    ffa = FFACUDA(cfg)
    t = ffa.autotune(e, v, reps=1)
    assert t["candidates"] > 3 and t["score_ms"] == 0.0 and t["bf_ms"] > 0.0
    got = ffa.execute(e, v)
    np.testing.assert_array_equal(got.view(np.uint32), lko.ffa(op, e, v).view(np.uint32))
    assert ffa.status() == 0


def test_multi_series_slots_identical(cuda):
    """Batches alternating over two executor slots (own streams, own graphs)
    give exactly the one-slot results; device inputs, several batches per
    length, partial last batches."""
    from loki_b200.batched import MultiSeriesSearch

    t = cuda
    rng = np.random.default_rng(8)
    lengths = [8192] * 7 + [5000] * 3 + [16384] * 4
    data = [(t.from_numpy(rng.standard_normal(L).astype(np.float32)).cuda(),
             t.from_numpy((1.0 + 0.2 * rng.random(L)).astype(np.float32)).cuda()) for L in lengths]
    kw = dict(tsamp=1e-3, nbins=32, f_range=(5.0, 9.0), widths=[1, 2, 3, 4], snr_min=3.0, max_batch=2)
    one = MultiSeriesSearch(n_slots=1, **kw).search(data)
    two = MultiSeriesSearch(n_slots=2, **kw).search(data)
    again = MultiSeriesSearch(n_slots=2, **kw)
    again.search(data[:3])
    three = again.search(data)  # graphs captured, slots reused
    tuned = MultiSeriesSearch(n_slots=2, autotune=True, **kw).search(data)  # launch shapes only
    for a, b, c, d in zip(one, two, three, tuned):
        for r in (b, c, d):
            assert r["total"] == a["total"] and r["nsamps"] == a["nsamps"]
            np.testing.assert_array_equal(r["idx"], a["idx"])
            np.testing.assert_array_equal(r["snr"].view(np.uint32), a["snr"].view(np.uint32))
    assert sum(r["total"] for r in one) > 0


# Valid-length batches: segments holding only padding are skipped by the
# brute fold (groups of 8 segments) and their folds set to +0.0, so folds and
# scores are bit-identical to folding the zeros. Lengths cover a full series,
# a partial last segment, fewer valid segments than one group, one sample and
# none. Shapes: two rows per warp in shared memory, with TMEM warps, and one
# row per warp (which folds everything).
LEN_CASES = {
    "accel_nb32_pk": (1 << 17, 1e-3, 32, ((-300.0, 300.0), (5.0, 8.0)), None),
    "accel_nb32_tmem": (1 << 17, 1e-3, 32, ((-300.0, 300.0), (5.0, 8.0)), (2, 6, 8)),
    "freq_nb128_tmem": (1 << 18, 64e-6, 128, ((20.0, 40.0),), (2, 4, 8)),
    "freq_nb128_rows1": (1 << 18, 64e-6, 128, ((20.0, 40.0),), (1, 8, 0)),
}


@pytest.mark.parametrize("name", sorted(LEN_CASES))
def test_batch_lengths_skip_padding(cuda, name):
    from loki_b200.ffa import FFACUDA

    t = cuda
    n, tsamp, nbins, lims, shape = LEN_CASES[name]
    cfg = _cfg(n, nbins, lims, tsamp=tsamp)
    lengths = [n, int(0.6 * n) + 37, int(0.13 * n), 1, 0]
    nb = len(lengths)
    plain = FFACUDA(cfg, max_batch=nb)
    skip = FFACUDA(cfg, max_batch=nb)
    if shape is not None:
        rows, ws, tw = shape
        tu = skip.tuning
        tu.update(bf_rows=rows, bf_warps=ws + tw, bf_tmem_warps=tw)
        skip.set_tuning(tu)
        plain.set_tuning(tu)
    es = np.zeros((nb, n), np.float32)
    vs = np.zeros((nb, n), np.float32)
    for k, L in enumerate(lengths):
        e, v = series(n, 60 + k)
        es[k, :L], vs[k, :L] = e[:L], v[:L]
    e = t.from_numpy(es).cuda()
    v = t.from_numpy(vs).cuda()
    lens = t.tensor(lengths, dtype=t.int64, device="cuda")
    skip.set_batch_lengths(lens)
    want_f = plain.execute_batch(e, v).cpu().numpy()
    want = plain.scores_batch(e, v).cpu().numpy()
    got = skip.scores_batch(e, v).cpu().numpy()
    nan = np.isnan(want)
    np.testing.assert_array_equal(np.isnan(got), nan)
    np.testing.assert_array_equal(got[~nan].view(np.uint32), want[~nan].view(np.uint32))
    got_f = skip.execute_batch(e, v).cpu().numpy()
    np.testing.assert_array_equal(got_f.view(np.uint32), want_f.view(np.uint32))
    # a captured step sees lengths (and data) written after the capture
    idx = t.empty(1 << 16, dtype=t.int32, device="cuda")
    snr = t.empty(1 << 16, dtype=t.float32, device="cuda")
    cnt = t.zeros(1, dtype=t.int64, device="cuda")
    thr = float(np.nanquantile(want, 0.999))
    skip.search_batch(e, v, thr, idx, snr, cnt)
    t.cuda.synchronize()
    g = t.cuda.CUDAGraph()
    with t.cuda.graph(g):
        skip.search_batch(e, v, thr, idx, snr, cnt)
    lengths2 = [0, n, 3, int(0.3 * n), n // 2]
    es2 = np.zeros((nb, n), np.float32)
    vs2 = np.zeros((nb, n), np.float32)
    for k, L in enumerate(lengths2):
        e2, v2 = series(n, 80 + k)
        es2[k, :L], vs2[k, :L] = e2[:L], v2[:L]
    e.copy_(t.from_numpy(es2))
    v.copy_(t.from_numpy(vs2))
    lens.copy_(t.tensor(lengths2, dtype=t.int64))
    g.replay()
    t.cuda.synchronize()
    k_n = int(cnt.item())
    flat = plain.scores_batch(e, v).cpu().numpy().ravel()
    want_idx = np.flatnonzero(flat >= thr)
    assert k_n == want_idx.size
    np.testing.assert_array_equal(idx[:k_n].cpu().numpy().view(np.uint32), want_idx.astype(np.uint32))
    np.testing.assert_array_equal(snr[:k_n].cpu().numpy().view(np.uint32), flat[want_idx].view(np.uint32))
    del g
    assert skip.status() == 0
