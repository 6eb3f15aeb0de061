"""Frequency sweep on the GPU (FFAFreqSweepCUDA): the chunk plan, per-chunk
FFA + scores + ordered `>= snr_min` compaction and the parameter decode,
through the C ABI, against the reference's whole sweeps (golden fixtures:
the reference planner, the reference FFA and scores per chunk, save_results'
decode) bit for bit, and against the oracle's sweep composition on a larger
chunked search."""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import golden, series
from oracle import sweep as osweep

pytestmark = pytest.mark.gpu

RUN_CASES = ["sweep_freq_2p16.npz", "sweep_accel_2p16.npz", "sweep_jerk_2p15.npz"]


def _cfg(g, snr_min=None):
    from loki_b200.configs import PulsarSearchConfig

    return PulsarSearchConfig(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                              np.asarray(g["param_limits"], np.float64), use_fourier=False,
                              max_process_memory_gb=float(g["max_memory_gb"]),
                              max_passing_candidates=int(g["max_passing"]),
                              snr_min=float(g["snr_min"]) if snr_min is None else snr_min)


@pytest.mark.parametrize("name", RUN_CASES)
@pytest.mark.parametrize("storage", ["fp32", "bf16"])
def test_sweep_matches_reference_fixture(cuda, name, storage):
    from loki_b200.sweep import FFAFreqSweepCUDA

    g = golden(name)
    for tag, cw in (("base_widths", False), ("chunk_widths", True)):
        sw = FFAFreqSweepCUDA(_cfg(g), fold_storage=storage, decode_chunk_widths=cw)
        mine = np.array([[c["f_min"], c["f_max"], c["nbins"], c["eta"]] for c in sw.chunks])
        np.testing.assert_array_equal(mine, g["chunks"][:, :4])
        params, snr = sw.run(g["ts_e"], g["ts_v"])
        np.testing.assert_array_equal(sw.region_counts, g["region_counts"])
        np.testing.assert_array_equal(params, g[f"params_{tag}"])
        np.testing.assert_array_equal(snr.view(np.uint32), g[f"snr_{tag}"].view(np.uint32))


@pytest.mark.parametrize("executors,autotune", [("resident", False), ("one_at_a_time", False),
                                                ("resident", True), ("one_at_a_time", True)])
def test_sweep_executor_modes_identical(cuda, executors, autotune):
    """Chunk executors kept on the device (chunks on two streams) or one chunk
    at a time (each executor released after its chunk): the reference's
    results either way, over two sweeps in a row."""
    from loki_b200.sweep import FFAFreqSweepCUDA

    g = golden("sweep_freq_2p16.npz")
    sw = FFAFreqSweepCUDA(_cfg(g), executors=executors, autotune=autotune)
    for _ in range(2):
        params, snr = sw.run(g["ts_e"], g["ts_v"])
        np.testing.assert_array_equal(sw.region_counts, g["region_counts"])
        np.testing.assert_array_equal(params, g["params_base_widths"])
        np.testing.assert_array_equal(snr.view(np.uint32), g["snr_base_widths"].view(np.uint32))


def test_sweep_execute_writes_results(cuda, tmp_path):
    from loki_b200 import libculoki

    g = golden("sweep_accel_2p16.npz")
    cfg = _cfg(g)
    sw = libculoki.ffa.FFAFreqSweepCUDA(cfg)
    path = sw.execute(g["ts_e"], g["ts_v"], str(tmp_path), "beam0")
    assert os.path.basename(path) == "beam0_ffa_results.npz"
    r = np.load(path)
    assert r["param_names"].tolist() == ["accel", "freq", "width"]
    np.testing.assert_array_equal(r["scoring_widths"], cfg.score_widths)
    np.testing.assert_array_equal(r["param_sets"], g["params_base_widths"])
    np.testing.assert_array_equal(r["snr"], g["snr_base_widths"])
    np.testing.assert_array_equal(r["region_counts"], g["region_counts"])
    # a second execute on the same sweep gives the same results
    p2, s2 = sw.run(g["ts_e"], g["ts_v"])
    np.testing.assert_array_equal(p2, g["params_base_widths"])


def test_sweep_device_inputs_and_threshold_rounding(cuda):
    """Device-tensor inputs; a threshold that is not a float: the candidate
    set is `float(score) >= snr_min` in double precision."""
    from loki_b200.sweep import FFAFreqSweepCUDA

    t = cuda
    g = golden("sweep_freq_2p16.npz")
    snr_min = float(np.nextafter(np.float32(6.5), np.float32(0))) + 1e-12  # strictly between two floats
    assert float(np.float32(snr_min)) != snr_min
    cfg = _cfg(g, snr_min=snr_min)
    sw = FFAFreqSweepCUDA(cfg)
    e = t.from_numpy(g["ts_e"]).cuda()
    v = t.from_numpy(g["ts_v"]).cuda()
    params, snr = sw.run(e, v)
    o_params, o_snr, _ = osweep.run((cfg.nsamps, cfg.tsamp, cfg.nbins, cfg.eta, g["param_limits"]),
                                    g["chunks"][:, :4], g["ts_e"], g["ts_v"], snr_min)
    np.testing.assert_array_equal(params, o_params)
    np.testing.assert_array_equal(snr.view(np.uint32), o_snr.view(np.uint32))
    assert np.all(snr.astype(np.float64) >= snr_min)


def test_sweep_larger_chunked_vs_oracle(cuda):
    """An accelerated search of 2^18 samples over 4-120 Hz whose regions are
    cut into several chunks each, against the oracle composition on the same
    chunk list (which the planner tests pin to the reference)."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.sweep import FFAFreqSweepCUDA

    nsamps, tsamp = 1 << 18, 256e-6
    lims = [[-40.0, 40.0], [4.0, 120.0]]
    ts_e, ts_v = series(nsamps, 77)
    tt = np.arange(nsamps) * tsamp
    for f0 in (9.3, 41.7, 88.8):
        ts_e += (0.35 * (np.mod(tt * f0, 1.0) < 0.04)).astype(np.float32)
    cfg = PulsarSearchConfig(nsamps, tsamp, 32, 2.0, np.array(lims), use_fourier=False,
                             max_process_memory_gb=0.514, max_passing_candidates=1 << 16, snr_min=7.0)
    sw = FFAFreqSweepCUDA(cfg, decode_chunk_widths=True)
    assert sw.nregions >= 8
    params, snr = sw.run(ts_e, ts_v)
    rows = np.array([[c["f_min"], c["f_max"], c["nbins"], c["eta"]] for c in sw.chunks])
    o_params, o_snr, o_counts = osweep.run((nsamps, tsamp, 32, 2.0, lims), rows, ts_e, ts_v, 7.0,
                                           chunk_widths=True)
    np.testing.assert_array_equal(sw.region_counts, o_counts)
    np.testing.assert_array_equal(params, o_params)
    np.testing.assert_array_equal(snr.view(np.uint32), o_snr.view(np.uint32))
    assert snr.size > 0
    # the injected signals are found at their frequencies
    for f0 in (9.3, 41.7, 88.8):
        assert np.any(np.abs(params[:, 1] - f0) < 0.05 * f0)


def test_sweep_octaves_to_nbins_max_vs_oracle(cuda):
    """A plain period sweep over 1-250 Hz whose octaves grow from 62 to the
    1024-bin cap (the brute fold's widest accumulators, the generic merge and
    scoring paths), against the oracle composition."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.sweep import FFAFreqSweepCUDA

    nsamps, tsamp = 1 << 17, 64e-6
    lims = [[1.0, 250.0]]
    ts_e, ts_v = series(nsamps, 5)
    tt = np.arange(nsamps) * tsamp
    for f0 in (2.3, 37.0, 180.0):
        ts_e += (0.3 * (np.mod(tt * f0, 1.0) < 0.03)).astype(np.float32)
    cfg = PulsarSearchConfig(nsamps, tsamp, 64, 1.0, np.array(lims), use_fourier=False,
                             max_passing_candidates=1 << 16, snr_min=6.0)
    for storage in ("fp32", "bf16"):
        sw = FFAFreqSweepCUDA(cfg, fold_storage=storage, decode_chunk_widths=True)
        assert [int(c["nbins"]) for c in sw.chunks] == [62, 124, 248, 496, 992, 1024]
        params, snr = sw.run(ts_e, ts_v)
        rows = np.array([[c["f_min"], c["f_max"], c["nbins"], c["eta"]] for c in sw.chunks])
        o_params, o_snr, o_counts = osweep.run((nsamps, tsamp, 64, 1.0, lims), rows, ts_e, ts_v, 6.0,
                                               chunk_widths=True)
        np.testing.assert_array_equal(sw.region_counts, o_counts)
        np.testing.assert_array_equal(params, o_params)
        np.testing.assert_array_equal(snr.view(np.uint32), o_snr.view(np.uint32))
        assert snr.size > 0


def test_fourier_sweep_vs_oracle(cuda):
    """The sweep with use_fourier = true (the reference default): chunks of the
    Fourier-domain planner, each through the Fourier-domain FFA (direct
    transform at 32 and 64 bins, the lossy level 0 at 128), against the FP64
    oracle chunk by chunk: every candidate whose FP64 S/N clears snr_min by the
    Fourier tolerance is found, nothing below it by that tolerance is, and
    every S/N agrees within it."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.sweep import FFAFreqSweepCUDA, FFARegionPlannerFourier

    nsamps, tsamp, snr_min = 1 << 17, 64e-6, 6.0
    lims = [[4.0, 70.0]]
    ts_e, ts_v = series(nsamps, 91)
    tt = np.arange(nsamps) * tsamp
    for f0 in (5.7, 21.3, 55.5):
        ts_e += (0.3 * (np.mod(tt * f0, 1.0) < 0.03)).astype(np.float32)
    cfg = PulsarSearchConfig(nsamps, tsamp, 32, 1.0, np.array(lims), max_passing_candidates=1 << 16,
                             snr_min=snr_min)  # use_fourier defaults to true
    sw = FFAFreqSweepCUDA(cfg, decode_chunk_widths=True)
    plan = FFARegionPlannerFourier(cfg, use_gpu=True)
    rows = np.array([[c["f_min"], c["f_max"], c["nbins"], c["eta"]] for c in sw.chunks])
    np.testing.assert_array_equal(rows, np.array([[c["f_min"], c["f_max"], c["nbins"], c["eta"]]
                                                  for c in plan.chunks]))
    assert {32, 64, 128} <= {int(r[2]) for r in rows}
    params, snr = sw.run(ts_e, ts_v)
    counts = np.asarray(sw.region_counts, np.int64)
    off = np.concatenate([[0], np.cumsum(counts)])
    lims0 = np.asarray(lims, np.float64)
    for i, (f_min, f_max, nb, eta) in enumerate(rows):
        lo = lims0.copy()
        lo[-1] = (f_min, f_max)
        s64, pc, w = osweep.lko_fourier_backend(nsamps, tsamp, int(nb), float(eta), lo, ts_e, ts_v)
        tol = 1e-3 + 5e-5 * np.abs(s64)
        sure = np.flatnonzero(s64 >= snr_min + tol)
        maybe = np.flatnonzero(s64 >= snr_min - tol)
        got = params[off[i]:off[i + 1]]
        got_snr = snr[off[i]:off[i + 1]].astype(np.float64)
        want_sure = osweep.decode(sure, pc, lo, w)
        want_maybe = osweep.decode(maybe, pc, lo, w)
        as_set = lambda a: {tuple(r) for r in a.tolist()}
        assert as_set(want_sure) <= as_set(got) <= as_set(want_maybe)
        # S/N of each candidate against the FP64 value of the same cell
        lookup = {tuple(r): s64[k] for r, k in zip(want_maybe.tolist(), maybe)}
        ref = np.array([lookup[tuple(r)] for r in got.tolist()])
        assert np.all(np.abs(got_snr - ref) <= 1e-3 + 5e-5 * np.abs(ref))
    assert snr.size > 0
    for f0 in (5.7, 21.3, 55.5):
        assert np.any(np.abs(params[:, 0] - f0) < 0.05 * f0)
