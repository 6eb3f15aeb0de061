"""GPU parity of the FFA path against the oracle (and, through the golden
fixtures, against the reference's own code). Every comparison is bit-exact:
coordinates, brute fold, final fold and boxcar scores."""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import golden, series
from oracle import lko

pytestmark = pytest.mark.gpu

# name -> (nsamps, tsamp, nbins, eta, param_limits, bseg_brute)
CASES = {
    "freq_nb64": (2**18, 64e-6, 64, 1.0, [[5.0, 50.0]], None),
    "freq_nb128": (2**19, 64e-6, 128, 1.0, [[20.0, 60.0]], None),
    "freq_nb100_generic": (2**18, 64e-6, 100, 1.0, [[10.0, 30.0]], None),
    "freq_nb16": (2**16, 64e-6, 16, 1.0, [[30.0, 60.0]], None),
    "freq_nb8": (2**16, 64e-6, 8, 1.0, [[30.0, 60.0]], None),
    "freq_nseg8": (2**14, 64e-6, 32, 1.0, [[100.0, 200.0]], 2048),
    "accel_nb64": (2**20, 64e-6, 64, 2.0, [[-200.0, 200.0], [5.0, 50.0]], None),
    "accel_multi_nb32": (2**18, 1e-3, 32, 1.0, [[-300.0, 300.0], [5.0, 8.0]], None),
    "accel_multi_nb64": (2**18, 1e-3, 64, 2.0, [[-200.0, 200.0], [5.0, 10.0]], None),
    "jerk_nb32": (2**19, 64e-6, 32, 2.0, [[-30.0, 30.0], [-3000.0, 3000.0], [20.0, 40.0]], None),
    "jerk_multi_nb32": (2**19, 5e-4, 32, 1.0, [[-50.0, 50.0], [-500.0, 500.0], [5.0, 7.0]], None),
}
WIDTHS = [1, 2, 3, 4, 6]


def make(name, widths=None):
    from loki_b200.configs import PulsarSearchConfig

    nsamps, tsamp, nbins, eta, lims, bseg = CASES[name]
    w = widths if widths is not None else [x for x in WIDTHS if x < nbins]
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, eta, np.array(lims), use_fourier=False, bseg_brute=bseg,
                             score_widths=w)
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims, bseg_brute=bseg))
    return cfg, op, np.array(w, dtype=np.uint64)


@pytest.mark.parametrize("name", sorted(CASES))
def test_coords_bit_exact(cuda, name):
    from loki_b200.plans import FFAPlanTime

    cfg, op, _ = make(name)
    got = FFAPlanTime(cfg).resolve_coordinates_flat()
    want = lko.resolve(op)
    assert got.tobytes() == want.tobytes()


@pytest.mark.parametrize("name", sorted(CASES))
def test_brute_fold_bit_exact(cuda, name):
    from loki_b200.fold import compute_brute_fold_time_cuda

    cfg, op, _ = make(name)
    ts_e, ts_v = series(cfg.nsamps, 11)
    got = compute_brute_fold_time_cuda(ts_e, ts_v, op.freqs0(), int(op.segment_lens[0]), cfg.nbins, cfg.tsamp,
                                       op.t_ref0())
    want = lko.brute_fold(ts_e, ts_v, op.freqs0(), int(op.segment_lens[0]), cfg.nbins, cfg.tsamp, op.t_ref0())
    assert got.shape == want.shape
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("seglen", [4, 16, 96, 160])
def test_brute_fold_short_and_partial_segments(cuda, seglen):
    """Segment lengths that are not whole 64-sample stages or 32-sample words."""
    from loki_b200.fold import compute_brute_fold_time_cuda

    n = seglen * 40
    ts_e, ts_v = series(n, 31 + seglen)
    freqs = np.linspace(90.0, 400.0, 13)
    got = compute_brute_fold_time_cuda(ts_e, ts_v, freqs, seglen, 16, 1e-3, 0.0)
    want = lko.brute_fold(ts_e, ts_v, freqs, seglen, 16, 1e-3, 0.0)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_brute_fold_misaligned_and_rebound_inputs(cuda):
    """Series views that are not 16-byte aligned go through an aligned copy;
    switching between input buffers rebinds the tensor maps."""
    from loki_b200.fold import BruteFoldCUDA

    t = cuda
    cfg, op, _ = make("accel_multi_nb32")
    n = cfg.nsamps
    seglen = int(op.segment_lens[0])
    bf = BruteFoldCUDA(op.freqs0(), seglen, cfg.nbins, n, cfg.tsamp, op.t_ref0())
    for seed, offset in ((21, 1), (22, 0), (23, 3)):
        ts_e, ts_v = series(n, seed)
        be = t.zeros(n + 4, dtype=t.float32, device="cuda")
        bv = t.zeros(n + 4, dtype=t.float32, device="cuda")
        be[offset:offset + n] = t.from_numpy(ts_e).cuda()
        bv[offset:offset + n] = t.from_numpy(ts_v).cuda()
        got = bf.execute(be[offset:offset + n], bv[offset:offset + n]).cpu().numpy()
        want = lko.brute_fold(ts_e, ts_v, op.freqs0(), seglen, cfg.nbins, cfg.tsamp, op.t_ref0())
        np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_ffa_fold_and_scores_bit_exact(cuda, name):
    from loki_b200.ffa import FFACUDA

    cfg, op, widths = make(name)
    ts_e, ts_v = series(cfg.nsamps, 12)
    ffa = FFACUDA(cfg)
    fold = ffa.execute(ts_e, ts_v)
    want = lko.ffa(op, ts_e, ts_v)
    np.testing.assert_array_equal(fold.view(np.uint32), want.view(np.uint32))
    if op.nsegments[-1] == 1:
        scores = ffa.scores(ts_e, ts_v)
        want_s = lko.snr_boxcar_3d(want, widths, cfg.nbins).ravel()
        np.testing.assert_array_equal(scores.view(np.uint32), want_s.view(np.uint32))
    assert ffa.status() == 0


@pytest.mark.parametrize("name", ["freq_nb64", "accel_multi_nb32", "jerk_multi_nb32"])
def test_search_matches_ordered_compaction(cuda, name):
    from loki_b200.ffa import FFACUDA

    cfg, op, widths = make(name)
    ts_e, ts_v = series(cfg.nsamps, 13)
    scores = lko.snr_boxcar_3d(lko.ffa(op, ts_e, ts_v), widths, cfg.nbins).ravel()
    thr = float(np.quantile(scores, 0.995))
    want_idx, want_val = lko.compact(scores, thr)
    idx, val, total = FFACUDA(cfg).search(ts_e, ts_v, snr_min=thr)
    assert total == want_idx.size
    np.testing.assert_array_equal(idx, want_idx)
    np.testing.assert_array_equal(val.view(np.uint32), want_val.view(np.uint32))


@pytest.mark.parametrize("name", ["ffa_freq_nb32.npz", "ffa_freq_nb64.npz", "ffa_accel_nb16.npz",
                                  "ffa_jerk_nb16.npz"])
def test_reference_golden_fixtures(cuda, name):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA
    from loki_b200.plans import FFAPlanTime

    g = golden(name)
    cfg = PulsarSearchConfig(int(g["nsamps"]), float(g["tsamp"]), int(g["nbins"]), float(g["eta"]),
                             g["param_limits"], use_fourier=False, score_widths=g["widths"].tolist())
    coords = FFAPlanTime(cfg).resolve_coordinates_flat()
    np.testing.assert_array_equal(coords.view(np.uint32).reshape(coords.size, -1), g["coords"])
    ffa = FFACUDA(cfg)
    fold = ffa.execute(g["ts_e"], g["ts_v"])
    assert hashlib.sha256(fold.tobytes()).hexdigest() == str(g["fold_sha256"])
    scores = ffa.scores(g["ts_e"], g["ts_v"])
    np.testing.assert_array_equal(scores.view(np.uint32), g["scores"].ravel().view(np.uint32))


def test_reference_golden_brute_fold(cuda):
    from loki_b200.fold import compute_brute_fold_time_cuda

    g = golden("brute_fold_nb64.npz")
    out = compute_brute_fold_time_cuda(g["ts_e"], g["ts_v"], g["freqs"], int(g["segment_len"]), int(g["nbins"]),
                                       float(g["tsamp"]), float(g["t_ref"]))
    np.testing.assert_array_equal(out.view(np.uint32), g["fold"].view(np.uint32))


def test_device_tensors_and_repeat_calls(cuda):
    from loki_b200.ffa import FFACUDA

    cfg, op, widths = make("accel_multi_nb32")
    ts_e, ts_v = series(cfg.nsamps, 14)
    ffa = FFACUDA(cfg)
    e = cuda.from_numpy(ts_e).cuda()
    v = cuda.from_numpy(ts_v).cuda()
    s1 = ffa.scores(e, v)
    s2 = ffa.scores(e, v)
    assert s1.is_cuda
    cuda.cuda.synchronize()
    assert cuda.equal(s1, s2)
    want = lko.snr_boxcar_3d(lko.ffa(op, ts_e, ts_v), widths, cfg.nbins).ravel()
    np.testing.assert_array_equal(s1.cpu().numpy().view(np.uint32), want.view(np.uint32))
    fold = cuda.zeros(ffa.plan.fold_size + 7, device="cuda")
    ffa.execute(e, v, fold)
    np.testing.assert_array_equal(fold[: ffa.plan.fold_size].cpu().numpy().view(np.uint32),
                                  lko.ffa(op, ts_e, ts_v).view(np.uint32))


def test_errors_are_loud(cuda):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA, compute_ffa_scores_cuda

    cfg, _, _ = make("freq_nb64")
    ffa = FFACUDA(cfg)
    with pytest.raises(RuntimeError, match="nsamps"):
        ffa.execute(np.zeros(100, np.float32), np.zeros(100, np.float32))
    fourier = PulsarSearchConfig(2**18, 64e-6, 64, 1.0, np.array([[5.0, 50.0]]))  # use_fourier default
    with pytest.raises(RuntimeError, match="nsamps"):
        compute_ffa_scores_cuda(np.zeros(100, np.float32), np.ones(100, np.float32), fourier)
    partial = PulsarSearchConfig(2**18, 64e-6, 64, 1.0, np.array([[5.0, 50.0]]), use_fourier=False,
                                 bseg_ffa=2**16)
    with pytest.raises(RuntimeError, match="nsegments must be 1"):
        FFACUDA(partial).scores(np.zeros(2**18, np.float32), np.ones(2**18, np.float32))


# Brute fold with part of the accumulators in tensor memory (TMEM warps):
# same sums in the same order, so folds stay bit-exact. Cases cover run bins
# stepping by one (nbins 16 / 32 / 64 / 128) and the bin-table path
# (frequencies above 1 / (tsamp nbins)), up to 256 bins (one column block of
# 512 TMEM columns per four warps).
TMEM_CASES = {
    "accel_nb64": (4, 8),
    "accel_multi_nb32": (6, 12),
    "freq_nb16": (2, 16),
    "freq_nb64_nonseq": (8, 4),
    "freq_nb128": (4, 8),
    "freq_nb128_nonseq": (6, 4),
    "freq_nb256_nonseq": (2, 4),
}
CASES_EXTRA = {
    "freq_nb64_nonseq": (2**17, 1e-3, 64, 1.0, [[20.0, 30.0]], None),
    "freq_nb128_nonseq": (2**17, 1e-3, 128, 1.0, [[20.0, 30.0]], None),
    "freq_nb256_nonseq": (2**18, 1e-3, 256, 1.0, [[3.0, 6.0]], None),
}


@pytest.mark.parametrize("name", sorted(TMEM_CASES))
def test_brute_fold_tmem_warps_bit_exact(cuda, name):
    from loki_b200.configs import PulsarSearchConfig
    from loki_b200.ffa import FFACUDA

    nsamps, tsamp, nbins, eta, lims, bseg = {**CASES, **CASES_EXTRA}[name]
    w = [x for x in WIDTHS if x < nbins]
    cfg = PulsarSearchConfig(nsamps, tsamp, nbins, eta, np.array(lims), use_fourier=False, bseg_brute=bseg,
                             score_widths=w)
    op = lko.plan_create(lko.make_cfg(nsamps, tsamp, nbins, eta, lims, bseg_brute=bseg))
    ts_e, ts_v = series(nsamps, 23)
    ffa = FFACUDA(cfg)
    ws, tw = TMEM_CASES[name]
    t = ffa.tuning
    t.update(bf_rows=2, bf_warps=ws + tw, bf_tmem_warps=tw)
    ffa.set_tuning(t)
    assert ffa.tuning["bf_tmem_warps"] == tw
    want = lko.ffa(op, ts_e, ts_v)
    got = ffa.execute(ts_e, ts_v)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
    want_s = lko.snr_boxcar_3d(want, np.array(w, np.uint64), nbins).ravel()
    got_s = ffa.scores(ts_e, ts_v)
    # cells whose variance sum is zero score NaN on both sides (0 / 0); only
    # the NaN's payload differs (x86 default NaN against the GPU's), so NaNs
    # are compared as NaN and every other score bit for bit
    nan = np.isnan(want_s)
    np.testing.assert_array_equal(np.isnan(got_s), nan)
    np.testing.assert_array_equal(got_s[~nan].view(np.uint32), want_s[~nan].view(np.uint32))
    assert ffa.status() == 0
