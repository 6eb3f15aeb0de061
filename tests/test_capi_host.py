"""The native library on the CPU: it loads, exports every entry point the
header declares, and its host-side plan logic (no GPU work) matches the
oracle -- and through it the reference -- exactly."""

from __future__ import annotations

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from oracle import lko

HEADER = os.path.join(ROOT, "include", "loki_b200.h")


def declared_symbols() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lk_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from loki_b200 import _capi

    lib = ctypes.CDLL(_capi.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each of them
    bound = {n for n, _, _ in _capi.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


CASES = [
    (2**21, 64e-6, 128, 1.0, [[5.0, 50.0]], None),
    (2**22, 64e-6, 64, 2.0, [[-200.0, 200.0], [5.0, 50.0]], None),
    (2**22, 64e-6, 64, 1.0, [[-200.0, 200.0], [5.0, 50.0]], None),
    (2**23, 64e-6, 32, 1.0, [[-0.4, 0.4], [-457.0, 457.0], [20.0, 200.0]], 2**18),
    (2**18, 64e-6, 128, 1.0, [[2.0, 50.0]], None),
    (2**20, 64e-6, 100, 1.5, [[10.0, 30.0]], None),
    (16384, 8e-3, 16, 1.0, [[-1000.0, 1000.0], [10.0, 10.3]], None),
]


@pytest.mark.parametrize("case", CASES)
def test_plan_geometry_matches_oracle(case):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.plans import FFAPlanTime

    nsamps, tsamp, nbins, eta, lims, bseg_ffa = case
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, eta, np.array(lims), use_fourier=False, bseg_ffa=bseg_ffa)
    plan = FFAPlanTime(cfg)
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims, bseg_ffa=bseg_ffa))
    assert plan.n_levels == op.n_levels
    assert cfg.bseg_brute == op.raw.bseg_brute
    np.testing.assert_array_equal(plan.ncoords, op.ncoords)
    np.testing.assert_array_equal(plan.nsegments, op.nsegments)
    np.testing.assert_array_equal(plan.segment_lens, op.segment_lens)
    np.testing.assert_array_equal(plan.ncoords_offsets, op.ncoords_offsets)
    np.testing.assert_array_equal(np.array(plan.param_counts), op.param_counts)
    assert np.array_equal(np.array(plan.dparams).view(np.uint64), op.dparams.view(np.uint64))
    assert plan.buffer_size == op.buffer_size
    assert plan.coord_size == op.coord_size
    np.testing.assert_array_equal(cfg.score_widths, op.widths)
    # brute-fold frequencies: range_param of level 0 (lib/ffa.cpp:177)
    f0 = plan.compute_param_grid(0)[-1]
    assert np.array_equal(f0.view(np.uint64), op.freqs0().view(np.uint64))


def test_config_properties_and_dparams():
    from loki_b200.configs import PulsarSearchConfig

    cfg = PulsarSearchConfig(2**22, 64e-6, 64, 2.0, np.array([[-200.0, 200.0], [5.0, 50.0]]), use_fourier=False)
    assert cfg.nparams == 2 and cfg.param_names == ["accel", "freq"]
    assert cfg.f_min == 5.0 and cfg.f_max == 50.0
    assert cfg.bseg_brute == 16384 and cfg.bseg_ffa == 2**22 and cfg.niters_ffa == 8
    assert cfg.tobs == pytest.approx(2**22 * 64e-6)
    assert cfg.nbins_f == 33
    op = lko.plan_create(lko.make_cfg(2**22, 64e-6, 64, 2.0, [[-200.0, 200.0], [5.0, 50.0]]))
    tseg = 16384 * 64e-6
    assert np.array_equal(cfg.dparams(tseg).view(np.uint64), op.dparams[0].view(np.uint64))
    act = cfg.dparams_actual(tseg)
    np.testing.assert_allclose(act, [400.0 / op.param_counts[0][0], 45.0 / op.param_counts[0][1]], rtol=0)
    upd = cfg.get_updated_config(128, 1.0, np.array([[-100.0, 100.0], [10.0, 20.0]]))
    assert upd.nbins == 128 and upd.f_min == 10.0


def test_explicit_score_widths():
    from loki_b200.configs import PulsarSearchConfig

    cfg = PulsarSearchConfig(2**21, 64e-6, 128, 1.0, np.array([[5.0, 50.0]]), score_widths=[1, 2, 3, 4, 6, 8, 12, 16])
    np.testing.assert_array_equal(cfg.score_widths, [1, 2, 3, 4, 6, 8, 12, 16])
    cfg2 = PulsarSearchConfig(2**21, 64e-6, 128, 1.0, np.array([[5.0, 50.0]]))
    np.testing.assert_array_equal(cfg2.score_widths, [1, 2, 3, 4, 6, 9, 13, 19])


@pytest.mark.parametrize(
    "kwargs, msg",
    [
        (dict(nsamps=3000), "power of 2"),
        (dict(tsamp=0.0), "tsamp must be positive"),
        (dict(eta=0.0), "eta"),
        (dict(bseg_brute=3000), "bseg_brute must be a power of 2"),
        (dict(bseg_brute=2**20), "bseg_brute must be less than nsamps"),
        (dict(param_limits=np.array([[50.0, 5.0]])), "increasing"),
        (dict(score_widths=[1, 200]), "score widths"),
    ],
)
def test_config_errors_raise(kwargs, msg):
    from loki_b200.configs import PulsarSearchConfig

    args = dict(nsamps=2**20, tsamp=64e-6, nbins=64, eta=1.0, param_limits=np.array([[5.0, 50.0]]))
    args.update(kwargs)
    with pytest.raises(RuntimeError, match=msg):
        PulsarSearchConfig(**args)


def test_width_trials_match_reference_fixture():
    from loki_b200.scores import generate_box_width_trials

    g = golden("scores_nb48.npz")
    np.testing.assert_array_equal(generate_box_width_trials(64, 0.2, 1.5), g["trials_64"])
    np.testing.assert_array_equal(generate_box_width_trials(128, 0.2, 1.5), g["trials_128"])
    np.testing.assert_array_equal(generate_box_width_trials(100, 0.3, 1.5), g["trials_100_03"])


def test_params_dict_and_fold_shapes():
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.plans import FFAPlanTime

    cfg = PulsarSearchConfig(2**20, 64e-6, 64, 2.0, np.array([[-200.0, 200.0], [5.0, 50.0]]), use_fourier=False)
    plan = FFAPlanTime(cfg)
    d = plan.params_dict
    assert list(d) == ["accel", "freq"]
    assert d["freq"].size == plan.param_counts[-1][1]
    shp = plan.fold_shapes[-1]
    assert shp.tolist() == [plan.nsegments[-1], *plan.param_counts[-1].tolist(), 2, 64]
    assert plan.fold_size == int(np.prod(shp))
    strides = plan.param_cart_strides[-1]
    assert strides.tolist() == [plan.param_counts[-1][1], 1]
