"""Hand-computed known answers for the oracle (the reference ships no golden
vectors; these restate the cases its own unit tests and code comments fix)."""

from __future__ import annotations

import numpy as np

from oracle import lko


def test_circular_prefix_sum_wraps():
    # tests/cpp/utils_t.cpp:53-80 of the reference.
    x = np.array([1, 2, 3, 4, 5], dtype=np.float32)
    np.testing.assert_array_equal(lko.circular_prefix_sum(x, 5), [1, 3, 6, 10, 15])
    np.testing.assert_array_equal(lko.circular_prefix_sum(x, 10), [1, 3, 6, 10, 15, 16, 18, 21, 25, 30])
    np.testing.assert_array_equal(lko.circular_prefix_sum(x, 3), [1, 3, 6])
    # second wrap: out[i] = out[i % n] + (i // n) * total (lib/utils.cpp:58-66)
    np.testing.assert_array_equal(lko.circular_prefix_sum(x, 12)[10:], [31, 33])


def test_brute_fold_period_of_four_samples():
    # f = 0.25 Hz at tsamp = 1 s: phase bin of sample i is i mod 4 (nbins 4).
    nbins, seglen = 4, 8
    x = np.arange(16, dtype=np.float32)
    v = np.ones(16, dtype=np.float32)
    fold = lko.brute_fold(x, v, [0.25], seglen, nbins, 1.0).reshape(2, 1, 2, nbins)
    for s in range(2):
        seg = x[s * seglen : (s + 1) * seglen]
        np.testing.assert_array_equal(fold[s, 0, 0], seg[:4] + seg[4:])
        np.testing.assert_array_equal(fold[s, 0, 1], [2, 2, 2, 2])


def test_brute_fold_half_up_rounding_and_wrap():
    # f = 0.3 Hz, nbins 4: iphase = frac(0.3 i) * 4 = 0, 1.2, 2.4, 3.6, 0.8,
    # 2.0, 3.2, 0.4, 1.6, 2.8 rounded half-up, 4 -> 0 (lib/loki/psr_utils.hpp:53-63).
    bins = [lko.phase_idx_uint(float(i), 0.3, 4) for i in range(10)]
    assert bins == [0, 1, 2, 0, 1, 2, 3, 0, 2, 3]
    x = np.arange(1, 11, dtype=np.float32)
    fold = lko.brute_fold(x, np.ones(10, np.float32), [0.3], 10, 4, 1.0)
    expect = np.zeros(4, dtype=np.float32)
    for i, b in enumerate(bins):
        expect[b] += x[i]
    np.testing.assert_array_equal(fold[:4], expect)


def test_phase_idx_edges():
    assert lko.phase_idx(0.0, 10.0, 64) == 0.0
    assert lko.phase_idx(-0.25, 1.0, 32) == 24.0       # negative time wraps into [0, nbins)
    assert lko.phase_idx(1.0, 1.0, 32, delay=0.5) == 16.0
    # 63.6 rounds half-up to 64 == nbins -> bin 0
    assert lko.phase_idx_uint(63.6 / 64.0, 1.0, 64) == 0


def test_merge_shift_of_nbins_wraps_to_zero():
    # shift phase 7.6 rounds to 8 == nbins -> no rotation (lib/kernels.cpp:42-49).
    nbins = 8
    fold = np.arange(2 * 2 * nbins, dtype=np.float32)  # [2 segments, 1 coord, 2, nbins]
    coords = np.zeros(1, dtype=lko.COORD_FREQ_DTYPE)
    coords["idx"] = 0
    coords["shift"] = 7.6
    out = lko.merge_freq(fold, coords, 1, 1, 1, nbins)
    np.testing.assert_array_equal(out, fold[:16] + fold[16:])
    coords["shift"] = 1.49  # rotate right by 1
    out = lko.merge_freq(fold, coords, 1, 1, 1, nbins)
    head = fold[16:].reshape(2, nbins)
    np.testing.assert_array_equal(out.reshape(2, nbins), fold[:16].reshape(2, nbins) + np.roll(head, 1, axis=1))


def test_merge_taylor_rotates_both_halves():
    nbins = 8
    rng = np.random.default_rng(0)
    fold = rng.standard_normal(2 * 3 * 2 * nbins).astype(np.float32)  # [2 seg, 3 coords, 2, nbins]
    coords = np.zeros(2, dtype=lko.COORD_DTYPE)
    coords[0] = (2, 3.0, 1, 5.2)
    coords[1] = (0, 0.4, 2, 7.7)
    out = lko.merge_taylor(fold, coords, 2, 3, 1, nbins).reshape(2, 2, nbins)
    f = fold.reshape(2, 3, 2, nbins)
    np.testing.assert_array_equal(out[0], np.roll(f[0, 2], 3, axis=1) + np.roll(f[1, 1], 5, axis=1))
    np.testing.assert_array_equal(out[1], np.roll(f[0, 0], 0, axis=1) + np.roll(f[1, 2], 0, axis=1))


def test_box_width_trials():
    # generate_box_width_trials (lib/score.cpp:390-405): nbins 128 -> {1,2,3,4,6,9,13,19}
    np.testing.assert_array_equal(lko.box_widths(128), [1, 2, 3, 4, 6, 9, 13, 19])
    np.testing.assert_array_equal(lko.box_widths(64), [1, 2, 3, 4, 6, 9])


def test_snr_of_a_flat_profile_is_zero_and_boxcar_is_matched():
    nbins = 32
    widths = np.array([1, 2, 4, 8], dtype=np.uint64)
    flat = np.zeros((1, 2, nbins), dtype=np.float32)
    flat[0, 0] = 3.0
    flat[0, 1] = 1.0
    s = lko.snr_boxcar_3d(flat, widths, nbins)
    np.testing.assert_allclose(s, 0.0, atol=1e-5)
    pulse = np.zeros((1, 2, nbins), dtype=np.float32)
    pulse[0, 1] = 1.0
    pulse[0, 0, 10:14] = 1.0  # width-4 boxcar: matched S/N = sqrt(4 (n-4)/n)
    s = lko.snr_boxcar_3d(pulse, widths, nbins)
    assert int(np.argmax(s[0])) == 2
    np.testing.assert_allclose(s[0, 2], np.sqrt(4 * (nbins - 4) / nbins), rtol=1e-6)


def test_compaction_keeps_ge_in_order():
    s = np.array([5.0, 4.9, 5.1, 7.0, 5.0, -1.0], dtype=np.float32)
    idx, val = lko.compact(s, 5.0)
    np.testing.assert_array_equal(idx, [0, 2, 3, 4])
    np.testing.assert_array_equal(val, s[[0, 2, 3, 4]])
