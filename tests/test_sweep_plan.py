"""Frequency-sweep planning and decode, CPU side.

The native region planner (octave regions, memory-bounded chunking by
bisection with drift-widened frequency ranges; the reference's
FFARegionPlanner, lib/regions.cpp) against the reference's own chunk plans
(golden fixtures made by tests/golden/make_golden.py from the reference build,
and -- where oracle/_ref is built -- the live reference planner on further
configurations), bit for bit; and the oracle's sweep composition (C-oracle FFA
+ scores + compaction + save_results decode) against the reference's whole
sweeps. Planning touches no device."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import ref as R
from oracle import sweep as osweep

PLAN_CASES = ["accel_2p22_8gb_cpu", "accel_2p22_8gb_gpu", "freq_2p22_2gb_gpu", "jerk_2p20_3gb_cpu",
              "freq_2p16_tight_gpu", "freq_2p16_tight_cpu", "accel_2p16_tight_gpu", "jerk_2p15_tight_gpu"]
RUN_CASES = ["sweep_freq_2p16.npz", "sweep_accel_2p16.npz", "sweep_jerk_2p15.npz"]


def _planner(nsamps, tsamp, nbins, eta, lims, mem, mp, gpu):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.sweep import FFARegionPlannerTime

    cfg = PulsarSearchConfig(int(nsamps), float(tsamp), int(nbins), float(eta), np.asarray(lims, np.float64),
                             use_fourier=False, max_process_memory_gb=float(mem),
                             max_passing_candidates=int(mp))
    return FFARegionPlannerTime(cfg, use_gpu=bool(gpu))


def _check_plan(p, rows, stats):
    ch = p.chunks
    assert len(ch) == rows.shape[0]
    mine = np.array([[c["f_min"], c["f_max"], c["nbins"], c["eta"]] for c in ch]).reshape(-1, 4)
    np.testing.assert_array_equal(mine, rows[:, :4])
    # bseg_brute / bseg_ffa of each chunk configuration (defaults recomputed per chunk)
    cfgs = p.get_cfgs()
    np.testing.assert_array_equal([c.bseg_brute for c in cfgs], rows[:, 4])
    np.testing.assert_array_equal([c.bseg_ffa for c in cfgs], rows[:, 5])
    ms = p.max_sizes
    assert [ms["max_buffer_size"], ms["max_coord_size"], ms["max_ncoords"], ms["max_ffa_levels"]] == \
        stats[:4].tolist()
    assert np.float32(ms["freq_sweep_memory_usage"]) == np.float32(stats[4])
    # chunks tile each region's nominal range from the top down
    for a, b in zip(ch, ch[1:]):
        if a["nbins"] == b["nbins"]:
            assert b["nominal_f_end"] == a["nominal_f_start"]
    assert all(c["allocated_gb"] <= float(p._cfg.max_process_memory_gb) - 0.5 for c in ch)


@pytest.mark.parametrize("name", PLAN_CASES)
def test_planner_matches_reference_fixture(name):
    g = golden("sweep_plans.npz")
    nsamps, tsamp, nbins, eta, mem, mp, gpu = g[f"{name}__inputs"]
    p = _planner(nsamps, tsamp, nbins, eta, g[f"{name}__lims"], mem, mp, gpu)
    _check_plan(p, g[f"{name}__rows"], g[f"{name}__stats"])


def _random_cases(n, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        npar = int(rng.integers(1, 4))
        nsamps = int(2 ** rng.integers(15, 23))
        tsamp = float(rng.choice([64e-6, 128e-6, 1e-3]))
        nbins = int(rng.choice([16, 32, 48, 64]))
        eta = float(rng.choice([1.0, 2.0, 3.0]))
        f_lo = float(rng.uniform(0.5, 20.0))
        f_hi = min(f_lo * float(rng.uniform(3.0, 200.0)), 0.2 / tsamp)
        lims = [[f_lo, f_hi]]
        if npar >= 2:
            a = float(rng.uniform(5.0, 300.0))
            lims.insert(0, [-a, a])
        if npar == 3:
            j = float(rng.uniform(0.5, 30.0))
            lims.insert(0, [-j, j])
        mem = float(rng.choice([0.52, 0.6, 1.0, 3.0, 8.0]))
        mp = int(rng.choice([4096, 1 << 20, 1 << 22]))
        out.append((nsamps, tsamp, nbins, eta, lims, mem, mp, bool(rng.integers(0, 2))))
    return out


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("case", _random_cases(24), ids=lambda c: f"np{len(c[4])}_n{c[0]}_m{c[5]}_g{int(c[7])}")
def test_planner_matches_live_reference(case):
    nsamps, tsamp, nbins, eta, lims, mem, mp, gpu = case
    try:
        rows, stats = R.region_plan(R.make_cfg(nsamps, tsamp, nbins, eta, lims), mem, 2.0, 1024, mp, gpu)
    except RuntimeError as e:
        # the reference refuses the configuration: so must the planner
        with pytest.raises(Exception):
            _planner(nsamps, tsamp, nbins, eta, lims, mem, mp, gpu)
        assert "FFARegionPlanner" in str(e) or "must" in str(e)
        return
    _check_plan(_planner(nsamps, tsamp, nbins, eta, lims, mem, mp, gpu), rows, stats)


def test_planner_refusals():
    from loki_b200 import _capi as C

    lims = [[-2.0, 2.0], [-20.0, 20.0], [2.0, 12.0]]
    with pytest.raises(C.LokiError, match="Cannot fit minimum viable chunk"):
        _planner(1 << 15, 2e-3, 16, 2.0, lims, 0.5015, 4096, False)
    with pytest.raises(C.LokiError, match="safety margin"):
        _planner(1 << 15, 2e-3, 16, 2.0, lims, 0.4, 4096, False)
    # a drift of a whole frequency (accel * T/2 / c >= 1) is refused
    with pytest.raises(C.LokiError, match="max_drift"):
        _planner(1 << 22, 1.0, 16, 2.0, [[-1e5, 1e5], [2.0, 12.0]], 8.0, 4096, False)


def test_generate_ffa_regions():
    from loki_b200.sweep import generate_ffa_regions

    r = generate_ffa_regions(1 / 500.0, 1 / 1.0, 64e-6, 64, 1.0)
    # octaves: nbins doubles with the period (first region capped at
    # p_min / tsamp samples), eta / nbins constant, last region at nbins_max
    assert r["nbins"].tolist() == [31, 62, 124, 248, 496, 992, 1024]
    np.testing.assert_allclose(r["eta"][:-1] / r["nbins"][:-1], 1.0 / 31.0)
    assert r["eta"][-1] == np.round(1024 / 31.0)
    assert r["f_end"][0] == 500.0 and r["f_start"][-1] == 1.0
    np.testing.assert_array_equal(r["f_start"][:-1], r["f_end"][1:])
    r2 = generate_ffa_regions(1 / 100.0, 1 / 10.0, 1e-4, 32, 2.0, growth_factor=1.5, nbins_max=64)
    assert r2["nbins"].max() == 64 and r2["nbins"][0] == 32
    from loki_b200 import _capi as C
    with pytest.raises(C.LokiError):
        generate_ffa_regions(1.0, 0.5, 1e-4, 32, 1.0)


@pytest.mark.parametrize("name", RUN_CASES)
def test_oracle_sweep_matches_reference_fixture(name):
    g = golden(name)
    base = (int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]), g["param_limits"])
    for tag, cw in (("base_widths", False), ("chunk_widths", True)):
        params, snr, counts = osweep.run(base, g["chunks"][:, :4], g["ts_e"], g["ts_v"], float(g["snr_min"]),
                                         chunk_widths=cw)
        np.testing.assert_array_equal(counts, g["region_counts"])
        np.testing.assert_array_equal(params, g[f"params_{tag}"])
        np.testing.assert_array_equal(snr.view(np.uint32), g[f"snr_{tag}"].view(np.uint32))
    assert g["snr_base_widths"].size > 0


def _planner_typed(nsamps, tsamp, nbins, eta, lims, mem, mp, gpu, fourier_plan, use_fourier):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.sweep import FFARegionPlannerFourier, FFARegionPlannerTime

    cfg = PulsarSearchConfig(int(nsamps), float(tsamp), int(nbins), float(eta), np.asarray(lims, np.float64),
                             use_fourier=use_fourier, max_process_memory_gb=float(mem),
                             max_passing_candidates=int(mp))
    cls = FFARegionPlannerFourier if fourier_plan else FFARegionPlannerTime
    return cls(cfg, use_gpu=bool(gpu))


@pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("fourier_plan,use_fourier", [(True, True), (False, True), (True, False)])
@pytest.mark.parametrize("case", _random_cases(10, seed=9), ids=lambda c: f"np{len(c[4])}_n{c[0]}_m{c[5]}")
def test_planner_fold_types_match_live_reference(case, fourier_plan, use_fourier):
    """FFARegionPlanner<ComplexType> / <float> on use_fourier configurations
    (fold buffers in harmonics or bins per row; 8-byte elements with
    use_fourier) against the reference's planner of the same fold type."""
    nsamps, tsamp, nbins, eta, lims, mem, mp, gpu = case
    try:
        rows, stats = R.region_plan(R.make_cfg(nsamps, tsamp, nbins, eta, lims), mem, 2.0, 1024, mp, gpu,
                                    complex_fold=fourier_plan, use_fourier=use_fourier)
    except RuntimeError:
        with pytest.raises(Exception):
            _planner_typed(nsamps, tsamp, nbins, eta, lims, mem, mp, gpu, fourier_plan, use_fourier)
        return
    _check_plan(_planner_typed(nsamps, tsamp, nbins, eta, lims, mem, mp, gpu, fourier_plan, use_fourier), rows,
                stats)
