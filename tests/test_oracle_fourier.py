"""Fourier-domain FFA: the C oracle (FP64) pinned to the reference.

* the direct transform of segments against numpy's matrix form of the same
  sum, and the real transforms against numpy.fft (FFTW's conventions: r2c
  unscaled, c2r scaled by 1 / n and blind to the imaginary parts of the DC
  and Nyquist terms);
* the oracle's level-0 transform, whole FFA (complex fold), fold back in
  time and boxcar S/N against the golden fixtures made by the reference's
  own FFA<ComplexType> (oracle/_ref, FP32), frequency, acceleration and jerk
  searches, and the lossy level 0 of nbins > 64. The reference sums and forms
  phasors in float, so the bar is a tolerance: folds within 2e-5 of the
  fold's largest magnitude, S/N within 1e-3;
* the same comparisons live against oracle/_ref where it is built.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import lko, ref

CASES = ["fourier_freq_nb32", "fourier_freq_nb64", "fourier_accel_nb16", "fourier_jerk_nb16",
         "fourier_freq_nb128_lossy"]
FOLD_RTOL = 2e-5   # of the fold's largest magnitude
SNR_ATOL = 1e-3
needs_ref = pytest.mark.skipif(not ref.available("parity"), reason="oracle/_ref not built")


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _plan(g):
    cfg = lko.make_cfg(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                       g["param_limits"])
    return lko.plan_create(cfg)


def test_direct_transform_matches_matrix_form():
    rng = np.random.default_rng(0)
    e = rng.standard_normal(3 * 512 + 100).astype(np.float32)
    v = (1 + 0.2 * rng.random(e.size)).astype(np.float32)
    freqs = np.array([7.3, 11.9, 49.95])
    tsamp, t_ref, L = 64e-6, 0.0171, 512
    for nb in (32, 33, 2):
        X = lko.fourier_brute_fold(e, v, freqs, L, nb, tsamp, t_ref)
        t = np.arange(L) * tsamp - t_ref
        m = np.arange(nb // 2 + 1)
        assert X.shape == (3, 3, 2, nb // 2 + 1)
        for s in range(3):
            for fi, f in enumerate(freqs):
                W = np.exp(-2j * np.pi * np.outer(m, f * t))
                np.testing.assert_allclose(X[s, fi, 0], W @ e[s * L:(s + 1) * L].astype(np.float64),
                                           rtol=1e-10, atol=1e-9)
                np.testing.assert_allclose(X[s, fi, 1], W @ v[s * L:(s + 1) * L].astype(np.float64),
                                           rtol=1e-10, atol=1e-9)


def test_real_transforms_follow_fftw_conventions():
    rng = np.random.default_rng(1)
    for n in (2, 16, 33, 64, 128):
        x = rng.standard_normal((4, n))
        np.testing.assert_allclose(lko.rfft(x, n), np.fft.rfft(x), atol=1e-9)
        np.testing.assert_allclose(lko.irfft(np.fft.rfft(x), n), x, atol=1e-12)
    z = np.fft.rfft(rng.standard_normal(32))
    zz = z.copy()
    zz[0] += 3j
    zz[-1] += 2j
    np.testing.assert_allclose(lko.irfft(zz, 32), np.fft.irfft(z, 32), atol=1e-12)


def test_merge_rotates_by_fractional_shift():
    rng = np.random.default_rng(2)
    nb, nbf = 16, 9
    fold = rng.standard_normal((2, 3, 2, nbf)) + 1j * rng.standard_normal((2, 3, 2, nbf))
    coords = np.zeros(2, dtype=lko.COORD_DTYPE)
    coords["i_tail"], coords["shift_tail"] = [0, 2], [0.25, 3.5]
    coords["i_head"], coords["shift_head"] = [1, 0], [15.75, 0.0]
    out = lko.fourier_merge(fold, coords, 2, 3, 1, nb)
    k = np.arange(nbf)
    for c in range(2):
        pt = np.exp(-2j * np.pi * k * coords["shift_tail"][c] / nb)
        ph = np.exp(-2j * np.pi * k * coords["shift_head"][c] / nb)
        want = fold[0, coords["i_tail"][c]] * pt + fold[1, coords["i_head"][c]] * ph
        np.testing.assert_allclose(out[0, c], want, atol=1e-12)


def test_brute_fold_matches_reference_fixture():
    g = golden("brute_fold_fourier.npz")
    for nb in (64, 33):
        X = lko.fourier_brute_fold(g["ts_e"], g["ts_v"], g["freqs"], int(g["segment_len"]), nb,
                                   float(g["tsamp"]), float(g["t_ref"]))
        assert _rel(X, g[f"fold_nb{nb}"]) < FOLD_RTOL


@pytest.mark.parametrize("name", CASES)
def test_ffa_matches_reference_fixture(name):
    g = golden(f"{name}.npz")
    p = _plan(g)
    assert p.n_levels == int(g["n_levels"])
    assert np.array_equal(p.ncoords, g["ncoords"])
    fold = lko.ffa_fourier(p, g["ts_e"], g["ts_v"])
    assert fold.size == int(g["fold_size"])
    nb = int(g["nbins"])
    if g["fold"].size:
        assert _rel(fold.ravel(), g["fold"]) < FOLD_RTOL
    if g["fold_time"].size:
        assert _rel(lko.irfft(fold, nb).ravel(), g["fold_time"]) < FOLD_RTOL
    assert np.array_equal(p.widths, g["widths"])
    s64 = lko.ffa_fourier_scores64(p, g["ts_e"], g["ts_v"], p.widths).ravel()
    assert np.abs(s64 - g["scores"]).max() < SNR_ATOL


@needs_ref
def test_ffa_matches_reference_live():
    rng = np.random.default_rng(3)
    n = 1 << 14
    e = rng.standard_normal(n).astype(np.float32)
    v = (1 + 0.25 * rng.random(n)).astype(np.float32)
    for lims, nb in (([[20.0, 40.0]], 64), ([[-500.0, 500.0], [12.0, 12.4]], 32)):
        lims = np.array(lims)
        rc = ref.make_cfg(n, 64e-6 if len(lims) == 1 else 4e-3, nb, 1.0, lims)
        oc = lko.make_cfg(n, 64e-6 if len(lims) == 1 else 4e-3, nb, 1.0, lims)
        p = lko.plan_create(oc)
        R = ref.RefFourier(rc)
        fold = lko.ffa_fourier(p, e, v)
        assert _rel(fold.ravel(), R.execute(e, v)) < FOLD_RTOL
        s = ref.fourier_scores(rc, e, v, int(p.ncoords[-1]) * p.widths.size)
        assert np.abs(lko.ffa_fourier_scores64(p, e, v, p.widths).ravel() - s).max() < SNR_ATOL


@needs_ref
@pytest.mark.parametrize("lims,nb", [([[20.0, 40.0]], 64), ([[-500.0, 500.0], [12.0, 12.4]], 32),
                                      ([[20.0, 40.0]], 128), ([[20.0, 40.0]], 33)])
def test_fourier_plan_geometry_matches_reference(lims, nb):
    """FFAPlanFourier (library, host only) against FFAPlan<ComplexType> of the reference."""
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.plans import FFAPlanFourier

    n, tsamp = 1 << 16, 64e-6 if len(lims) == 1 else 4e-3
    cfg = PulsarSearchConfig(n, tsamp, nb, 1.0, np.array(lims), use_fourier=True)
    p = FFAPlanFourier(cfg)
    R = ref.RefFourier(ref.make_cfg(n, tsamp, nb, 1.0, np.array(lims)))
    assert p.fold_size == R.fold_size
    assert p.buffer_size == R.buffer_size
    assert p.fold_size_time == R.fold_size_time
    assert p.buffer_size_time == 2 * R.buffer_size
    assert p.nbins_f == nb // 2 + 1
    assert [int(x) for x in p.fold_shapes[-1]][-1] == nb // 2 + 1
