"""GPU parity of the Fourier-domain FFA (FFACOMPLEXCUDA, the reference's
use_fourier = true path) against the FP64 oracle and, through the golden
fixtures, against the reference's own FFA<ComplexType>.

The path sums in FP32 with phasors from phases reduced in FP64, so the bar
is a tolerance written here: complex and back-in-time folds within
FOLD_RTOL of the fold's largest magnitude of the FP64 oracle, S/N within
SNR_ATOL + SNR_RTOL |S/N| of the oracle's FP64 S/N (an FP32 sum's error
grows with its value; the reference's own FP32 Fourier path sits up to
7e-5 |S/N| from FP64), and candidate sets equal to the oracle's except for
cells whose FP64 S/N lies within that tolerance of the threshold.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, series
from oracle import lko

pytestmark = pytest.mark.gpu

FOLD_RTOL = 2e-5
SNR_ATOL = 1e-3
SNR_RTOL = 5e-5


def _snr_ok(got, want):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    return bool(np.all(np.abs(got - want) <= SNR_ATOL + SNR_RTOL * np.abs(want)))
FIXTURES = ["fourier_freq_nb32", "fourier_freq_nb64", "fourier_accel_nb16", "fourier_jerk_nb16",
            "fourier_freq_nb128_lossy"]
# name -> (nsamps, tsamp, nbins, eta, param_limits)
CASES = {
    "freq_nb64_2p18": (2**18, 64e-6, 64, 1.0, [[10.0, 25.0]]),
    "freq_nb33_odd": (2**16, 64e-6, 33, 1.0, [[20.0, 40.0]]),
    "accel_nb64_2p18": (2**18, 64e-6, 64, 2.0, [[-200.0, 200.0], [20.0, 50.0]]),
    "accel_nb32_multi": (2**17, 1e-3, 32, 1.0, [[-300.0, 300.0], [5.0, 8.0]]),
    "jerk_nb32": (2**17, 5e-4, 32, 1.0, [[-50.0, 50.0], [-500.0, 500.0], [5.0, 7.0]]),
    "freq_nb128_lossy": (2**16, 64e-6, 128, 1.0, [[20.0, 40.0]]),
    "freq_nb256_lossy": (2**15, 64e-6, 256, 1.0, [[20.0, 30.0]]),
}


def _rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _make(nsamps, tsamp, nbins, eta, lims):
    from loki_b200.configs import PulsarSearchConfig

    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims))
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, eta, np.array(lims), use_fourier=True,
                             score_widths=[int(w) for w in op.widths])
    return cfg, op


def test_brute_fold_vs_fixture_and_oracle(cuda):
    from loki_b200.fold import compute_brute_fold_fourier_cuda

    g = golden("brute_fold_fourier.npz")
    for nb in (64, 33):
        got = compute_brute_fold_fourier_cuda(g["ts_e"], g["ts_v"], g["freqs"], int(g["segment_len"]), nb,
                                              float(g["tsamp"]), float(g["t_ref"]))
        want = lko.fourier_brute_fold(g["ts_e"], g["ts_v"], g["freqs"], int(g["segment_len"]), nb,
                                      float(g["tsamp"]), float(g["t_ref"]))
        assert _rel(got, want.ravel()) < FOLD_RTOL
        assert _rel(got, g[f"fold_nb{nb}"].ravel()) < 2 * FOLD_RTOL


def test_brute_fold_ragged_segments(cuda):
    from loki_b200.fold import compute_brute_fold_fourier_cuda

    ts_e, ts_v = series(5 * 1000 + 77, 3)  # 5 segments of 1000 (not a multiple of 256), tail dropped
    freqs = np.array([3.1, 17.77, 42.0])
    for nb in (2, 16, 64):
        got = compute_brute_fold_fourier_cuda(ts_e, ts_v, freqs, 1000, nb, 1e-3, 0.5)
        want = lko.fourier_brute_fold(ts_e, ts_v, freqs, 1000, nb, 1e-3, 0.5)
        assert got.size == want.size
        assert _rel(got, want.ravel()) < FOLD_RTOL


@pytest.mark.parametrize("name", FIXTURES)
def test_ffa_vs_reference_fixture(cuda, name):
    from loki_b200.ffa import FFACOMPLEXCUDA

    g = golden(f"{name}.npz")
    nb = int(g["nbins"])
    cfg, op = _make(int(g["nsamps"]), float(g["tsamp"]), nb, float(g["eta"]), g["param_limits"])
    ffa = FFACOMPLEXCUDA(cfg)
    assert ffa.lossy == (nb > 64)
    fold = ffa.execute(g["ts_e"], g["ts_v"])
    assert fold.size == int(g["fold_size"])
    want = lko.ffa_fourier(op, g["ts_e"], g["ts_v"]).ravel()
    assert _rel(fold, want) < FOLD_RTOL
    if g["fold"].size:
        assert _rel(fold, g["fold"]) < 2 * FOLD_RTOL
    tfold = ffa.execute_time(g["ts_e"], g["ts_v"])
    assert _rel(tfold, lko.irfft(want, nb).ravel()) < FOLD_RTOL
    if g["fold_time"].size:
        assert _rel(tfold, g["fold_time"]) < 2 * FOLD_RTOL
    s = ffa.scores(g["ts_e"], g["ts_v"])
    s64 = lko.ffa_fourier_scores64(op, g["ts_e"], g["ts_v"], op.widths).ravel()
    assert _snr_ok(s, s64)
    assert np.abs(s - g["scores"]).max() < 2 * SNR_ATOL


@pytest.mark.parametrize("name", sorted(CASES))
def test_ffa_vs_oracle(cuda, name):
    from loki_b200.ffa import FFACOMPLEXCUDA

    nsamps, tsamp, nb, eta, lims = CASES[name]
    cfg, op = _make(nsamps, tsamp, nb, eta, lims)
    ts_e, ts_v = series(nsamps, 17)
    ffa = FFACOMPLEXCUDA(cfg)
    fold = ffa.execute(ts_e, ts_v)
    want = lko.ffa_fourier(op, ts_e, ts_v).ravel()
    assert _rel(fold, want) < FOLD_RTOL
    s = ffa.scores(ts_e, ts_v)
    s64 = lko.ffa_fourier_scores64(op, ts_e, ts_v, op.widths).ravel()
    assert _snr_ok(s, s64)
    # candidate set of a threshold inside the S/N distribution
    thr = float(np.quantile(s64, 0.999))
    idx, snr, total = ffa.search(ts_e, ts_v, snr_min=thr, max_cands=1 << 20)
    assert total == idx.size
    assert np.all(np.diff(idx.astype(np.int64)) > 0)
    assert np.array_equal(snr, s[idx])
    tol = SNR_ATOL + SNR_RTOL * abs(thr)
    sure = np.flatnonzero(s64 >= thr + tol)
    maybe = np.flatnonzero(s64 >= thr - tol)
    assert np.isin(sure, idx).all() and np.isin(idx, maybe).all()


def test_device_tensors_and_dispatch(cuda):
    import torch

    from loki_b200.ffa import FFACOMPLEXCUDA, compute_ffa_fourier_cuda, compute_ffa_scores_cuda

    nsamps, tsamp, nb, eta, lims = CASES["accel_nb32_multi"]
    cfg, op = _make(nsamps, tsamp, nb, eta, lims)
    ts_e, ts_v = series(nsamps, 5)
    host, plan = compute_ffa_fourier_cuda(ts_e, ts_v, cfg)
    assert host.dtype == np.complex64 and host.size == plan.fold_size
    ffa = FFACOMPLEXCUDA(cfg)
    dev = ffa.execute(torch.from_numpy(ts_e).cuda(), torch.from_numpy(ts_v).cuda())
    assert dev.is_cuda and dev.dtype == torch.float32
    assert np.array_equal(dev.cpu().numpy().view(np.complex64), host)
    # the reference's overload pair: a float32 host buffer receives the fold in time
    buf = np.zeros(plan.buffer_size_time, dtype=np.float32)
    ffa.execute(ts_e, ts_v, buf)
    assert np.array_equal(buf[: plan.fold_size_time], ffa.execute_time(ts_e, ts_v))
    s, _ = compute_ffa_scores_cuda(ts_e, ts_v, cfg)  # use_fourier=True routes to the Fourier path
    assert np.array_equal(s, ffa.scores(ts_e, ts_v))


def test_profile_stages(cuda):
    from loki_b200.ffa import FFACOMPLEXCUDA

    nsamps, tsamp, nb, eta, lims = CASES["freq_nb128_lossy"]
    cfg, _ = _make(nsamps, tsamp, nb, eta, lims)
    ts_e, ts_v = series(nsamps, 6)
    ffa = FFACOMPLEXCUDA(cfg)
    ffa.set_profiling(True)
    ffa.scores(ts_e, ts_v)
    stages = [p["stage"] for p in ffa.profile()]
    assert stages[0] == "brute_fold" and stages[1] == "transform" and stages[-1] == "score"
    assert stages.count("merge") == ffa.plan.n_levels - 1


# level-0 shapes: (nsamps, tsamp, nbins, eta, limits, bseg_brute) -> tensor-core
# tiles of one subtile (few segments), two subtiles and several column groups
L0_CASES = {
    "nb64_few_segments": (2**14, 64e-6, 64, 1.0, [[20.0, 30.0]], None),
    "nb64_accel": (2**18, 64e-6, 64, 2.0, [[-200.0, 200.0], [20.0, 50.0]], None),
    "nb32_many_segments": (2**17, 64e-6, 32, 1.0, [[30.0, 60.0]], 256),
    "nb33_odd": (2**16, 64e-6, 33, 1.0, [[20.0, 40.0]], 1024),
    "nb16_1024_segments": (2**18, 1e-3, 16, 1.0, [[5.0, 8.0]], 256),
}


@pytest.mark.parametrize("name", sorted(L0_CASES))
def test_level0_tensor_cores_vs_cuda_cores(cuda, name):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACOMPLEXCUDA
    from loki_b200.fold import compute_brute_fold_fourier_cuda

    nsamps, tsamp, nb, eta, lims, bseg = L0_CASES[name]
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nb, eta, lims, bseg_brute=bseg))
    cfg = PulsarSearchConfig(nsamps, tsamp, nb, eta, np.array(lims), use_fourier=True, bseg_brute=bseg,
                             score_widths=[int(w) for w in op.widths])
    ts_e, ts_v = series(nsamps, 23)
    ts_e *= np.float32(37.5)  # not unit scale: the FP16 staging exponent is exercised
    final = lko.ffa_fourier(op, ts_e, ts_v).ravel()
    s64 = lko.ffa_fourier_scores64(op, ts_e, ts_v, op.widths).ravel()
    ffa = FFACOMPLEXCUDA(cfg)
    for mode in ("cuda_cores", "tensor_cores"):
        ffa.set_level0(mode)
        fold = ffa.execute(ts_e, ts_v)
        assert ffa.status() == 0
        assert _rel(fold, final) < FOLD_RTOL, mode
        s = ffa.scores(ts_e, ts_v)
        assert _snr_ok(s, s64), mode
    # level 0 alone through the brute-fold entry (the direct transform on the CUDA cores)
    want0 = lko.ffa_fourier(op, ts_e, ts_v, level=0).ravel()
    freqs = ffa.plan.compute_param_grid(0)[-1]
    t_ref = 0.0 if len(lims) == 1 else float(op.raw.tsegments[0]) / 2
    bf = compute_brute_fold_fourier_cuda(ts_e, ts_v, freqs, int(op.segment_lens[0]), nb, tsamp, t_ref)
    assert _rel(bf, want0) < FOLD_RTOL


def test_autotune_keeps_results(cuda):
    from loki_b200.ffa import FFACOMPLEXCUDA

    nsamps, tsamp, nb, eta, lims = CASES["accel_nb64_2p18"]
    cfg, op = _make(nsamps, tsamp, nb, eta, lims)
    ts_e, ts_v = series(nsamps, 31)
    ffa = FFACOMPLEXCUDA(cfg)
    assert ffa.level0 == "tensor_cores"
    before = ffa.scores(ts_e, ts_v)
    ms = ffa.autotune(ts_e, ts_v, reps=2)
    assert ms > 0
    after = ffa.scores(ts_e, ts_v)
    assert ffa.status() == 0
    s64 = lko.ffa_fourier_scores64(op, ts_e, ts_v, op.widths).ravel()
    assert _snr_ok(before, s64) and _snr_ok(after, s64)
