"""DynamicThresholdScheme: the C oracle (and the library's host set-up)
pinned to the reference.

* Philox4x32-10 against the published known-answer vectors (Random123);
* the normal quantile table against scipy's ndtri (the reference builds it
  with Boost.Math, absent here), entry for entry after rounding to float;
* thresholds, probabilities, the folded profile, the bound scheme,
  find_neighbouring_indices, find_lower_bin_index and State::gen_next
  against the reference's own functions (oracle/_ref), bit for bit;
* whole runs of the oracle against the golden fixtures made by restating
  the reference's stage loop over its own pieces, every State field bit for
  bit, and against that restatement live where oracle/_ref exists;
* get_best_path_thresholds of the reference on those states.
"""

from __future__ import annotations

import ast

import numpy as np
import pytest

from conftest import golden
from oracle import lko, ref

FIELDS = [f for f in lko.DTS_STATE_DTYPE.names if f != "_pad"]
needs_ref = pytest.mark.skipif(not ref.available("parity"), reason="oracle/_ref not built")


def _states_equal(a, b):
    for f in FIELDS:
        x, y = np.asarray(a[f]), np.asarray(b[f])
        if x.dtype == np.float32:
            x, y = x.view(np.uint32), y.astype(np.float32).view(np.uint32)
        if not np.array_equal(x, y):
            return False
    return True


def test_philox_known_answers():
    # Random123 known-answer vectors of philox4x32_10
    assert lko.philox4x32_10([0, 0, 0, 0], 0).tolist() == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert lko.philox4x32_10([0xFFFFFFFF] * 4, 0xFFFFFFFFFFFFFFFF).tolist() == [
        0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert lko.philox4x32_10([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                             (0x299F31D0 << 32) | 0xA4093822).tolist() == [0xD16CFE09, 0x94FDCCEB, 0x5001E420,
                                                                          0x24126EA1]


def test_normal_table_matches_scipy():
    from scipy.special import ndtri

    lut = lko.dts_normal_lut()
    p = np.clip(np.arange(lut.size, dtype=np.float64) / (lut.size - 1), 1e-9, 1 - 1e-9)
    np.testing.assert_array_equal(lut.view(np.uint32), ndtri(p).astype(np.float32).view(np.uint32))


def test_library_host_setup_matches_oracle():
    from loki_b200.thresholds import dts_plan, normal_lut

    np.testing.assert_array_equal(normal_lut().view(np.uint32), lko.dts_normal_lut().view(np.uint32))
    for ns, nbins, ducy, snr, nthr, npb, pmin, dmax, wtsp in [(8, 32, 0.1, 8.0, 50, 6, 0.05, 0.3, 1.0),
                                                              (30, 64, 0.05, 9.0, 100, 10, 0.02, 0.2, 1.5),
                                                              (12, 100, 0.2, 7.0, 64, 12, 0.1, 0.3, 1.0)]:
        bp = np.linspace(1.2, 6.0, ns).astype(np.float32)
        p = dts_plan(bp, ducy, nbins=nbins, nprobs=npb, prob_min=pmin, snr_final=snr, nthresholds=nthr,
                     ducy_max=dmax, wtsp=wtsp)
        np.testing.assert_array_equal(p["profile"].view(np.uint32), lko.dts_profile(nbins, ducy).view(np.uint32))
        np.testing.assert_array_equal(p["thresholds"], lko.dts_thresholds(0.1, snr, nthr))
        np.testing.assert_array_equal(p["probs"], lko.dts_probs(npb, pmin))
        np.testing.assert_array_equal(p["guess_path"], lko.dts_guess(ns, snr, bp))
        np.testing.assert_array_equal(p["widths"], lko.box_widths(nbins, dmax, wtsp).astype(np.uint32))


@needs_ref
def test_setup_pieces_match_reference():
    for snr, n in [(8.0, 100), (7.0, 60), (10.0, 37)]:
        np.testing.assert_array_equal(lko.dts_thresholds(0.1, snr, n).view(np.uint32),
                                      ref.dts_thresholds(0.1, snr, n).view(np.uint32))
    for n, pmin in [(10, 0.05), (8, 0.1), (25, 0.001)]:
        np.testing.assert_array_equal(lko.dts_probs(n, pmin).view(np.uint32), ref.dts_probs(n, pmin).view(np.uint32))
    for nbins, ducy, center in [(64, 0.1, 0.5), (32, 0.05, 0.5), (100, 0.2, 0.3), (128, 0.3, 0.9)]:
        np.testing.assert_array_equal(lko.dts_profile(nbins, ducy, center).view(np.uint32),
                                      ref.dts_profile(nbins, ducy, center).view(np.uint32))
    # the guess path is min(bound, trials); the bound part is the reference's
    for ns, snr in [(8, 8.0), (30, 9.0)]:
        bp = np.full(ns, 1.0, np.float32)  # trials stay at the 1e10 floor: norm_isf(1e-10) ~ 6.36
        g = lko.dts_guess(ns, snr, bp)
        b = ref.dts_bound(ns, snr)
        isf = np.float32(6.361340902404056)
        np.testing.assert_array_equal(g, np.minimum(b, np.float32(g.max())))
        assert abs(g.max() - isf) < 1e-6 or (g == b).all()


@needs_ref
def test_neighbours_lower_bin_gen_next_match_reference():
    rng = np.random.default_rng(3)
    for _ in range(200):
        n = int(rng.integers(1, 30))
        idx = np.unique(rng.integers(0, 100, n)).astype(np.uint32)
        t = int(rng.integers(0, 100))
        num = int(rng.integers(1, 15))
        np.testing.assert_array_equal(lko.dts_neighbours(idx, t, num), ref.dts_neighbours(idx, t, num))
    probs = lko.dts_probs(10, 0.05)
    for v in list(rng.random(200).astype(np.float32)) + [0.0, 0.04999, 1.0, float(probs[3])]:
        assert lko.dts_lower_bin(probs, v) == ref.dts_lower_bin(probs, v)
    st = np.zeros(1, lko.DTS_STATE_DTYPE)[0]
    for _ in range(100):
        for f in ("complexity", "complexity_cumul", "success_h1_cumul", "threshold"):
            st[f] = np.float32(rng.random() * 10)
        args = (np.float32(rng.random() * 8), np.float32(rng.random()), np.float32(rng.random()),
                np.float32(rng.random() * 6 + 1))
        want = ref.dts_gen_next(st, *args, lko.DTS_STATE_DTYPE)
        got = np.zeros(1, lko.DTS_STATE_DTYPE)
        assert want["is_empty"] == 0
        # the oracle's gen_next runs inside lko_dts_run; compare its formula here
        nl = np.float32(st["complexity"]) * args[3]
        assert want["complexity"] == np.float32(nl * args[1])
        assert want["complexity_cumul"] == np.float32(st["complexity_cumul"] + nl)
        assert want["success_h1_cumul"] == np.float32(st["success_h1_cumul"] * args[2])
        assert want["cost"] == np.float32(want["complexity_cumul"] / want["success_h1_cumul"])
        del got


@pytest.mark.parametrize("name", ["dts_nb32.npz", "dts_nb48.npz"])
def test_oracle_run_matches_reference_fixture(name):
    g = golden(name)
    kw = ast.literal_eval(str(g["config"][0]))
    bp = g["branching"]
    import hashlib

    assert hashlib.sha256(lko.dts_normal_lut().tobytes()).hexdigest() == str(g["lut_sha256"])
    np.testing.assert_array_equal(lko.dts_guess(bp.size, kw.get("snr_final", 8.0), bp), g["guess"])
    got = lko.dts_run(bp, float(g["ref_ducy"]), **kw)
    want = {f: g[f"state_{f}"] for f in FIELDS}
    assert _states_equal(got, want)
    assert (~got["is_empty"]).sum() > 50


@needs_ref
def test_oracle_run_matches_reference_live():
    bp = np.linspace(1.5, 4.0, 6).astype(np.float32)
    kw = dict(nbins=64, ntrials=200, nprobs=5, nthresholds=40, thres_neigh=3, beam_width=1.0, prob_min=0.1,
              seed=12345)
    a = lko.dts_run(bp, 0.1, **kw)
    b = ref.dts_run(bp, 0.1, lko.dts_guess(6, 8.0, bp), lko.dts_normal_lut(), lko.DTS_STATE_DTYPE, **kw)
    assert _states_equal(a, b)
