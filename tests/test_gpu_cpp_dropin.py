"""The C++20 drop-in classes (include/loki_b200.hpp: PulsarSearchConfig,
FFAPlan<float>, FFACUDA<float>, FFACUDA<ComplexTypeCUDA>,
compute_ffa_scores_cuda over the C ABI), compiled by build() into
tests/cpp/_build/ffacuda_check: the time-domain fold and scores bit-identical
to the oracle, the Fourier-domain fold and scores within the Fourier path's
tolerance of the FP64 oracle, and the reference's exception types on
rejected arguments."""

from __future__ import annotations

import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, series
from oracle import lko

pytestmark = pytest.mark.gpu

EXE = os.path.join(ROOT, "tests", "cpp", "_build", "ffacuda_check")


@pytest.mark.parametrize("case", [
    (1 << 17, 1e-3, 32, 1.0, [[-300.0, 300.0], [5.0, 8.0]], [1, 2, 3, 4, 6]),
    (1 << 18, 64e-6, 64, 1.0, [[20.0, 40.0]], [1, 2, 4, 8]),
])
def test_cpp_dropin_matches_oracle(cuda, tmp_path, case):
    if not os.path.exists(EXE):
        pytest.fail("tests/cpp/_build/ffacuda_check is missing: run __graft_entry__.build()")
    nsamps, tsamp, nbins, eta, lims, widths = case
    ts_e, ts_v = series(nsamps, 5)
    lim = np.asarray(lims, np.float64).ravel()
    with open(tmp_path / "in.bin", "wb") as fh:
        fh.write(np.array([nsamps], np.uint64).tobytes() + np.array([tsamp], np.float64).tobytes()
                 + np.array([nbins], np.uint64).tobytes() + np.array([eta], np.float64).tobytes()
                 + np.array([len(lims)], np.uint32).tobytes() + lim.tobytes()
                 + np.array([len(widths)], np.uint32).tobytes() + np.array(widths, np.uint32).tobytes()
                 + ts_e.tobytes() + ts_v.tobytes())
    r = subprocess.run([EXE, str(tmp_path / "in.bin"), str(tmp_path / "fold.bin"), str(tmp_path / "scores.bin"),
                        str(tmp_path / "cfold.bin"), str(tmp_path / "cscores.bin")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims))
    want_fold = lko.ffa(op, ts_e, ts_v)
    got_fold = np.fromfile(tmp_path / "fold.bin", np.float32)
    np.testing.assert_array_equal(got_fold.view(np.uint32), want_fold.view(np.uint32))
    want = lko.snr_boxcar_3d(want_fold, np.array(widths, np.uint64), nbins).ravel()
    got = np.fromfile(tmp_path / "scores.bin", np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    # Fourier-domain path (use_fourier = true)
    cfold = np.fromfile(tmp_path / "cfold.bin", np.complex64)
    want_c = lko.ffa_fourier(op, ts_e, ts_v).ravel()
    assert cfold.size == want_c.size
    assert np.abs(cfold - want_c).max() < 2e-5 * np.abs(want_c).max()
    cs = np.fromfile(tmp_path / "cscores.bin", np.float32)
    want_cs = lko.ffa_fourier_scores64(op, ts_e, ts_v, np.array(widths, np.uint64)).ravel()
    assert np.abs(cs - want_cs).max() < 1e-3
