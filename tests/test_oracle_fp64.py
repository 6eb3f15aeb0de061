"""The FP64 restatement of the FFA agrees with the FP32 oracle to FP32
rounding: folds within 1e-5 relative (of the row's scale), S/N within 1e-4."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import series
from oracle import fp64, lko

CASES = {
    "freq_nb32": (2**15, 64e-6, 32, 1.0, [[30.0, 60.0]]),
    "accel_nb32": (2**16, 1e-3, 32, 1.0, [[-300.0, 300.0], [5.0, 8.0]]),
}
WIDTHS = [1, 2, 3, 4, 6]


@pytest.mark.parametrize("name", sorted(CASES))
def test_fp64_ffa_matches_fp32_oracle(name):
    nsamps, tsamp, nbins, eta, lims = CASES[name]
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims))
    ts_e, ts_v = series(nsamps, 5)
    want = lko.ffa(op, ts_e, ts_v).reshape(-1, 2, nbins).astype(np.float64)
    got = fp64.ffa64(op, ts_e, ts_v).reshape(-1, 2, nbins)
    scale = np.abs(want).max(axis=2, keepdims=True) + 1.0
    assert np.max(np.abs(got - want) / scale) < 1e-5
    s32 = lko.snr_boxcar_3d(lko.ffa(op, ts_e, ts_v), np.array(WIDTHS, dtype=np.uint64), nbins)
    s64 = fp64.ffa_scores64(op, ts_e, ts_v, WIDTHS)
    assert np.max(np.abs(s64 - s32)) < 1e-4
