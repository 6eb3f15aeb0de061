"""BF16 fold storage (levels 1 .. L-2 in BF16, every add FP32).

Checks: (1) a BF16 search returns exactly the FP32 search's candidates
(indices, S/N bit patterns, totals), because every cell near the threshold is
rescored exactly; (2) the approximate BF16 scores stay well inside the
rescoring margin; (3) errors against the FP64 oracle: FP32 S/N within 1e-4,
BF16 candidates' S/N (exact rescored values) within 1e-3, BF16 all-cell S/N
within the stated rounding model; (4) FP16 storage is refused."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import series
from oracle import fp64, lko

pytestmark = pytest.mark.gpu

# name -> (nsamps, tsamp, nbins, eta, param_limits, pulsars (f0, accel, jerk, snr))
CASES = {
    "freq_nb64": (2**18, 64e-6, 64, 1.0, [[5.0, 50.0]], [(17.3, 0.0, 0.0, 14.0)]),
    "freq_nb128": (2**19, 64e-6, 128, 1.0, [[20.0, 60.0]], [(33.1, 0.0, 0.0, 11.0), (51.7, 0.0, 0.0, 25.0)]),
    "accel_nb64": (2**20, 64e-6, 64, 2.0, [[-200.0, 200.0], [5.0, 50.0]], [(23.4, 80.0, 0.0, 15.0)]),
    "accel_multi_nb32": (2**18, 1e-3, 32, 1.0, [[-300.0, 300.0], [5.0, 8.0]], [(6.1, -120.0, 0.0, 12.0)]),
    "jerk_nb32": (2**19, 64e-6, 32, 2.0, [[-30.0, 30.0], [-3000.0, 3000.0], [20.0, 40.0]],
                  [(31.0, 900.0, 5.0, 16.0)]),
}
WIDTHS = [1, 2, 3, 4, 6, 8]


def make(name, seed=41):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.synthetic import Pulsar, make_series

    nsamps, tsamp, nbins, eta, lims, psrs = CASES[name]
    w = [x for x in WIDTHS if x < nbins]
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, eta, np.array(lims), use_fourier=False, score_widths=w)
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims))
    pulsars = [Pulsar(f0=f, accel=a, jerk=j, snr=s) for f, a, j, s in psrs]
    ts_e, ts_v = make_series(nsamps, tsamp, seed, pulsars, nbins, w)
    # variance series with structure (the V rows are not all equal)
    ts_v = ts_v * (1.0 + 0.25 * np.random.default_rng(seed + 1).random(nsamps)).astype(np.float32)
    return cfg, op, w, ts_e, ts_v


@pytest.mark.parametrize("name", sorted(CASES))
def test_bf16_search_candidates_identical(cuda, name):
    from loki_b200.ffa import FFACUDA

    cfg, op, w, ts_e, ts_v = make(name)
    plain = FFACUDA(cfg, fold_storage="fp32")
    mixed = FFACUDA(cfg, fold_storage="bf16")
    assert plain.scores_exact and not mixed.scores_exact  # BF16 scores() are approximate
    s32 = plain.scores(ts_e, ts_v)
    for q in (0.99, 0.999, 0.99999):
        thr = float(np.quantile(s32, q))
        i32, v32, n32 = plain.search(ts_e, ts_v, snr_min=thr)
        i16, v16, n16 = mixed.search(ts_e, ts_v, snr_min=thr)
        assert n16 == n32
        np.testing.assert_array_equal(i16, i32)
        np.testing.assert_array_equal(v16.view(np.uint32), v32.view(np.uint32))
        ncells = mixed.rescored_cells()
        uniq = np.unique(i32 // len(w)).size
        assert uniq <= ncells < s32.size // len(w)
    assert mixed.status() == 0


@pytest.mark.parametrize("name", sorted(CASES))
def test_bf16_scores_within_margin_and_fp64_errors(cuda, name):
    from loki_b200.ffa import FFACUDA

    cfg, op, w, ts_e, ts_v = make(name)
    plain = FFACUDA(cfg, fold_storage="fp32")
    mixed = FFACUDA(cfg, fold_storage="bf16")
    s32 = plain.scores(ts_e, ts_v).reshape(-1, len(w)).astype(np.float64)
    s16 = mixed.scores(ts_e, ts_v).reshape(-1, len(w)).astype(np.float64)
    s64 = fp64.ffa_scores64(op, ts_e, ts_v, w)
    m_abs, m_rel = mixed.rescore_margin
    L = int(op.n_levels)
    assert m_abs > 0 and m_rel > 0
    # the margin is a bound on |approx - exact| with wide headroom
    err = np.abs(s16 - s32)
    assert np.all(err <= (m_abs + m_rel * np.abs(s32)) / 3.0), float(err.max())
    # FP32 path vs FP64: the plain form's S/N tolerance
    assert np.max(np.abs(s32 - s64)) < 1e-4
    # BF16 all-cell S/N vs FP64: RMS within 2x the rounding model
    u = 2.0**-8
    model = u * np.sqrt(max(L - 2, 1) / 3.0) + u / np.sqrt(3.0) * np.abs(s64)
    assert np.sqrt(np.mean((s16 - s64) ** 2)) < 2.0 * np.sqrt(np.mean(model**2))
    # candidates of a BF16 search carry exact FP32 S/N: within 1e-3 of FP64
    thr = float(np.quantile(s32, 0.999))
    idx, val, _ = mixed.search(ts_e, ts_v, snr_min=thr)
    assert idx.size > 0
    assert np.max(np.abs(val - s64.ravel()[idx])) < 1e-3


@pytest.mark.parametrize("name", ["freq_nb64", "accel_nb64"])
def test_bf16_fold_error(cuda, name):
    from loki_b200.ffa import FFACUDA

    cfg, op, w, ts_e, ts_v = make(name)
    f16 = FFACUDA(cfg, fold_storage="bf16").execute(ts_e, ts_v).reshape(-1, 2, cfg.nbins).astype(np.float64)
    f64 = fp64.ffa64(op, ts_e, ts_v).reshape(-1, 2, cfg.nbins)
    L = int(op.n_levels)
    # V rows are positive: relative error at most (L - 2) 2^-8 (first order)
    v_rel = np.abs(f16[:, 1] - f64[:, 1]) / f64[:, 1]
    assert v_rel.max() <= (L - 2) * 2.0**-8 * 1.01
    # E rows: error relative to the bin's noise scale sqrt(V)
    e_err = np.abs(f16[:, 0] - f64[:, 0]) / np.sqrt(f64[:, 1])
    assert np.sqrt(np.mean(e_err**2)) < 2.0 * 2.0**-8 * np.sqrt(max(L - 2, 1) / 3.0) * 4


def test_bf16_batch_candidates_identical(cuda):
    from loki_b200.ffa import FFACUDA

    t = cuda
    cfg, op, w, _, _ = make("accel_multi_nb32")
    ser = [make("accel_multi_nb32", seed=s)[3:] for s in (51, 52, 53)]
    e = t.from_numpy(np.stack([x[0] for x in ser])).cuda()
    v = t.from_numpy(np.stack([x[1] for x in ser])).cuda()
    plain = FFACUDA(cfg, fold_storage="fp32", max_batch=4)
    mixed = FFACUDA(cfg, fold_storage="bf16", max_batch=4)
    s32 = plain.scores_batch(e, v).cpu().numpy()
    thr = float(np.quantile(s32, 0.999))
    out = []
    for ex in (plain, mixed):
        idx = t.empty(1 << 16, dtype=t.int32, device="cuda")
        snr = t.empty(1 << 16, dtype=t.float32, device="cuda")
        cnt = t.zeros(1, dtype=t.int64, device="cuda")
        ex.search_batch(e, v, thr, idx, snr, cnt)
        n = int(cnt.item())
        out.append((idx[:n].cpu().numpy(), snr[:n].cpu().numpy()))
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))
    assert out[0][0].size > 0


def test_margin_api_and_fp16_refused(cuda):
    from loki_b200 import _capi as C
    from loki_b200.ffa import FFACUDA

    cfg, op, w, ts_e, ts_v = make("freq_nb64")
    mixed = FFACUDA(cfg, fold_storage="bf16")
    mixed.set_rescore_margin(0.5, 0.1)
    assert mixed.rescore_margin == (0.5, pytest.approx(0.1))
    with pytest.raises(C.LokiError):
        mixed.set_rescore_margin(-1.0, 0.0)
    plain = FFACUDA(cfg, fold_storage="fp32")
    assert plain.rescore_margin == (0.0, 0.0)
    with pytest.raises(C.LokiError):
        FFACUDA(cfg, fold_storage="fp16")


def _error_statement(nsamps: int):
    """FP32 and BF16-stored S/N and folds against the FP64 oracle on the
    accelerated-search workload (seed 7, four signals) at nsamps samples."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA
    from loki_b200.synthetic import Pulsar, make_series

    tsamp, nbins, eta = 64e-6, 64, 2.0
    lims = [[-200.0, 200.0], [5.0, 50.0]]
    widths = [1, 2, 3, 4, 6, 8, 12, 16]
    rng = np.random.default_rng(7 + 1000)
    psrs = [Pulsar(f0=float(rng.uniform(5, 50)), accel=float(rng.uniform(-150, 150)), duty=0.05,
                   snr=float(rng.uniform(8, 20))) for _ in range(4)]
    ts_e, ts_v = make_series(nsamps, tsamp, 7, psrs, nbins, widths)
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, eta, np.array(lims), use_fourier=False, score_widths=widths)
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims))
    plain = FFACUDA(cfg, fold_storage="fp32")
    mixed = FFACUDA(cfg, fold_storage="bf16")
    s64 = lko.ffa_scores64(op, ts_e, ts_v, np.array(widths, np.uint64)).ravel()
    s32 = plain.scores(ts_e, ts_v).astype(np.float64)
    s16 = mixed.scores(ts_e, ts_v).astype(np.float64)
    thr = 7.0
    i32, v32, n32 = plain.search(ts_e, ts_v, snr_min=thr)
    i16, v16, n16 = mixed.search(ts_e, ts_v, snr_min=thr)
    assert n16 == n32 and np.array_equal(i16, i32) and np.array_equal(v16.view(np.uint32), v32.view(np.uint32))
    e16 = s16 - s64
    stat = {
        "nsamps": nsamps, "cells": int(s64.size), "candidates": int(n32),
        "rescored_cells": mixed.rescored_cells(),
        "fp32_snr_max_abs_err": float(np.max(np.abs(s32 - s64))),
        "bf16_snr_rms_err": float(np.sqrt(np.mean(e16**2))),
        "bf16_snr_max_abs_err": float(np.max(np.abs(e16))),
        "bf16_snr_max_abs_err_at_or_above_6": float(np.max(np.abs(e16[s64 >= 6.0]))) if np.any(s64 >= 6.0) else 0.0,
        "candidate_snr_max_abs_err": float(np.max(np.abs(v16.astype(np.float64) - s64[i16]))) if n16 else 0.0,
        "margin": list(mixed.rescore_margin),
    }
    print("ERRSTAT", stat)
    assert stat["fp32_snr_max_abs_err"] < 1e-4
    assert stat["candidate_snr_max_abs_err"] < 1e-3
    return stat


def test_error_statement_accel_2p20(cuda):
    _error_statement(1 << 20)


def test_error_statement_accel_2p22(cuda):
    _error_statement(1 << 22)
