"""GPU boxcar scoring and compaction against the oracle (bit-exact)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from oracle import lko

pytestmark = pytest.mark.gpu


def folds3d(nprof, nbins, seed, pulse=True):
    rng = np.random.default_rng(seed)
    f = np.empty((nprof, 2, nbins), dtype=np.float32)
    f[:, 0] = rng.standard_normal((nprof, nbins)) * 8
    f[:, 1] = 64 + rng.random((nprof, nbins)) * 4
    if pulse:
        f[::7, 0, : max(1, nbins // 10)] += 40
    return f


@pytest.mark.parametrize("nbins, widths", [
    (8, [1, 2, 3]), (32, [1, 2, 3, 4, 6]), (48, [1, 2, 3, 5, 8, 13]), (64, [1, 2, 3, 4, 6, 8, 12, 16]),
    (100, [1, 2, 3, 4, 6, 9, 13, 19]), (128, [1, 2, 3, 4, 6, 8, 12, 16]), (256, [1, 2, 4, 8, 16, 32, 51]),
])
def test_snr_boxcar_3d_bit_exact(cuda, nbins, widths):
    from loki_b200 import scores as S

    f = folds3d(1000, nbins, nbins)
    w = np.array(widths, dtype=np.uint64)
    got = S.snr_boxcar_3d(f, w)
    np.testing.assert_array_equal(got.view(np.uint32), lko.snr_boxcar_3d(f, w, nbins).view(np.uint32))
    got_max = S.snr_boxcar_3d_max(f, w)
    np.testing.assert_array_equal(got_max.view(np.uint32), lko.snr_boxcar_3d_max(f, w, nbins).view(np.uint32))


def test_snr_boxcar_2d_max_bit_exact(cuda):
    from loki_b200 import scores as S

    rng = np.random.default_rng(3)
    prof = rng.standard_normal((777, 64)).astype(np.float32)
    w = np.array([1, 2, 3, 4, 6, 9], dtype=np.uint64)
    got = S.snr_boxcar_2d_max(prof, w, stdnoise=2.5)
    np.testing.assert_array_equal(got.view(np.uint32), lko.snr_boxcar_2d_max(prof, w, 64, 2.5).view(np.uint32))


def test_scores_golden_fixture(cuda):
    from loki_b200 import scores as S

    g = golden("scores_nb48.npz")
    np.testing.assert_array_equal(S.snr_boxcar_3d(g["folds"], g["widths"]).view(np.uint32),
                                  g["scores"].view(np.uint32))
    np.testing.assert_array_equal(S.snr_boxcar_3d_max(g["folds"], g["widths"]).view(np.uint32),
                                  g["scores_max"].view(np.uint32))


def test_scorer_rejects_bad_widths(cuda):
    from loki_b200 import scores as S

    with pytest.raises(RuntimeError, match="widths"):
        S.snr_boxcar_3d(folds3d(4, 16, 0), [1, 16])
    with pytest.raises(RuntimeError, match="empty"):
        S.snr_boxcar_3d(np.zeros((0, 2, 16), np.float32), [1])


@pytest.mark.parametrize("n", [1, 1000, 4096, 4097, 100_003, 3_000_000])
def test_compact_ge_matches_oracle(cuda, n):
    from loki_b200 import scores as S

    rng = np.random.default_rng(n)
    s = rng.standard_normal(n).astype(np.float32)
    s[::5] = 2.0  # exact ties at the threshold are kept (>=)
    idx, val, total = S.compact_ge(s, 2.0)
    wi, wv = lko.compact(s, 2.0)
    assert total == wi.size
    np.testing.assert_array_equal(idx, wi)
    np.testing.assert_array_equal(val.view(np.uint32), wv.view(np.uint32))


def test_compact_ge_edges(cuda):
    from loki_b200 import scores as S

    s = np.arange(10000, dtype=np.float32)
    idx, val, total = S.compact_ge(s, 1e9)
    assert total == 0 and idx.size == 0
    idx, val, total = S.compact_ge(s, -1.0)
    assert total == 10000 and np.array_equal(idx, np.arange(10000))
    idx, val, total = S.compact_ge(s, 5000.0, max_out=17)
    assert total == 5000 and np.array_equal(idx, np.arange(5000, 5017))
