"""Monte-Carlo threshold stage on the GPU against the C oracle (whose
per-profile decision is pinned to the reference's
snr_boxcar_threshold_with_cache in tests/test_oracle_mc.py): survivor folds,
survivor rows, grid counts and maximum S/N bit-exact, through a cascade."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lko

pytestmark = pytest.mark.gpu

WIDTHS = np.array([1, 2, 3, 4, 6, 8, 12, 16], np.uint32)


def oracle_cascade(folds0, signal, cls, noises, thresholds, grids):
    out, rows, fin, var = [], np.arange(folds0.shape[0], dtype=np.uint32), folds0, 1.0
    for s, nz in enumerate(noises):
        f, ids, counts, _ = lko.mc_stage(fin, nz, signal, var, var, WIDTHS.astype(np.uint64), thresholds[s],
                                         grids[s], signal_scale=float(2 ** s), rowmap=rows, cls=cls)
        g = len(grids[s])
        out.append({"alive": rows.size, "kept": ids.size, "counts": counts[:g], "counts_flagged": counts[g:],
                    "folds": f, "ids": ids})
        fin, rows, var = f, ids, 2 * var
        if rows.size == 0:
            break
    return out


def test_mc_cascade_bit_exact(cuda):
    from loki_b200.synthetic import mc_cascade_workload
    from loki_b200.thresholds import mc_cascade

    folds0, signal, cls, noises, thresholds, grids = mc_cascade_workload(ntrials=6000, nstages=4, seed=5)
    want = oracle_cascade(folds0, signal, cls, noises, thresholds, grids)
    got = mc_cascade(folds0, signal, noises, cls, WIDTHS, thresholds, grids)
    assert len(got) == len(want)
    for g, w in zip(got, want):
        assert (g["alive"], g["kept"]) == (w["alive"], w["kept"])
        np.testing.assert_array_equal(g["counts"].astype(np.uint64), w["counts"])
        np.testing.assert_array_equal(g["counts_flagged"].astype(np.uint64), w["counts_flagged"])
    assert 0 < got[-1]["kept"] < got[0]["alive"]


@pytest.mark.parametrize("per_trial", [False, True])
def test_mc_stage_folds_ids_and_max_snr(cuda, per_trial):
    from loki_b200.thresholds import MCStageCUDA

    rng = np.random.default_rng(17)
    n, nb = 3001, 48
    fin = rng.standard_normal((n, nb)).astype(np.float32)
    nz = rng.standard_normal((n + 50, nb)).astype(np.float32) * np.float32(1.3)
    sig = (rng.random((n + 50, nb)) if per_trial else rng.random(nb)).astype(np.float32)
    rows = rng.permutation(n + 50)[:n].astype(np.uint32)
    src = rng.integers(0, n, n).astype(np.uint32)
    widths = np.array([1, 2, 3, 5, 8, 13], np.uint32)
    grid = np.linspace(0.0, 6.0, 37).astype(np.float32)
    f_w, ids_w, counts_w, mx_w = lko.mc_stage(fin, nz, sig, 1.69, 1.69, widths.astype(np.uint64), 2.5, grid,
                                              src=src, signal_scale=4.0, rowmap=rows, ntrials=n)
    st = MCStageCUDA(n, nb, widths)
    r = st.stage(fin, nz, sig, 2.5, 1.69, 1.69, thresholds=grid, signal_scale=4.0, rowmap=rows, src=src,
                 ntrials=n, with_max_snr=True)
    k = int(r["count"].item())
    assert st.status() == 0
    assert k == ids_w.size and 0 < k < n
    np.testing.assert_array_equal(r["max_snr"].cpu().numpy(), mx_w)
    np.testing.assert_array_equal(r["folds"][:k].cpu().numpy(), f_w)
    np.testing.assert_array_equal(r["ids"][:k].cpu().numpy().view(np.uint32), ids_w)
    np.testing.assert_array_equal(r["counts"].cpu().numpy().astype(np.uint64), counts_w)


@pytest.mark.parametrize("grid_kind", ["sorted_ties", "shuffled", "with_nan"])
def test_mc_stage_grid_counts(cuda, grid_kind):
    """Grid counts (all trials and class-flagged ones) for a non-decreasing
    grid with repeated values (counted by rank), a shuffled grid and one with
    a NaN entry (counted per grid value), against the oracle."""
    from loki_b200.thresholds import MCStageCUDA

    rng = np.random.default_rng(23)
    n, nb = 4099, 64
    fin = rng.standard_normal((n, nb)).astype(np.float32)
    nz = rng.standard_normal((n, nb)).astype(np.float32)
    sig = rng.random(nb).astype(np.float32)
    cls = (rng.random(n) < 0.3).astype(np.uint8)
    grid = np.round(np.linspace(0.0, 8.0, 64), 1).astype(np.float32)
    grid[10:14] = grid[10]
    if grid_kind == "shuffled":
        grid = rng.permutation(grid)
    elif grid_kind == "with_nan":
        grid[20] = np.nan
    f_w, ids_w, counts_w, mx_w = lko.mc_stage(fin, nz, sig, 1.0, 1.0, WIDTHS.astype(np.uint64), 3.0, grid,
                                              signal_scale=2.0, cls=cls)
    st = MCStageCUDA(n, nb, WIDTHS)
    r = st.stage(fin, nz, sig, 3.0, 1.0, 1.0, thresholds=grid, signal_scale=2.0, cls=cls)
    np.testing.assert_array_equal(r["counts"].cpu().numpy().astype(np.uint64), counts_w)
    assert int(r["count"].item()) == ids_w.size


def test_mc_stage_reference_api_and_errors(cuda):
    from loki_b200 import LokiError
    from loki_b200.thresholds import MCStageCUDA, simulate_score_prune_fused

    rng = np.random.default_rng(3)
    n, nb = 1000, 32
    fin = rng.standard_normal((n, nb)).astype(np.float32)
    nz = rng.standard_normal((n, nb)).astype(np.float32)
    prof = np.exp(-0.5 * ((np.arange(nb) - 16) / 2.0) ** 2).astype(np.float32)
    out, frac = simulate_score_prune_fused(fin, prof, nz, 3.0, [1, 2, 4, 8], var_in=1.0, bias_snr=2.0)
    f_w, _, _, _ = lko.mc_stage(fin, nz, (prof * np.float32(2.0)).astype(np.float32), 1.0, 1.0,
                                np.array([1, 2, 4, 8], np.uint64), 3.0)
    np.testing.assert_array_equal(out, f_w)
    assert frac == f_w.shape[0] / n
    st = MCStageCUDA(n, nb, [1, 2, 4, 8])
    with pytest.raises(LokiError, match="max_trials"):
        st.stage(fin, np.zeros((2 * n, nb), np.float32), prof, 3.0, 1.0, 1.0, ntrials=2 * n)
    with pytest.raises(LokiError, match="64 thresholds"):
        st.stage(fin, nz, prof, 3.0, 1.0, 1.0, thresholds=np.zeros(65, np.float32))
    # a row index beyond the noise rows is caught by the kernel's bounds check
    bad = np.arange(n, dtype=np.uint32)
    bad[7] = 10 * n
    st.stage(fin, nz, prof, 3.0, 1.0, 1.0, rowmap=bad)
    assert st.status() != 0
    assert st.status() == 0
