"""Generates the golden fixtures in this folder from the reference's own code.

Run from the repository root after ``make -C oracle ref``:

    python tests/golden/make_golden.py          # every fixture
    python tests/golden/make_golden.py prune    # the pruning fixtures only
    python tests/golden/make_golden.py sweep    # the frequency-sweep fixtures only
    python tests/golden/make_golden.py dts      # the threshold-scheme fixtures only
    python tests/golden/make_golden.py fourier  # the Fourier-domain FFA fixtures only

Every output comes from ``oracle/_ref/libloki_ref_parity.so`` -- the
reference's CPU sources compiled unmodified with IEEE flags -- so the fixtures
pin both the C oracle and the CUDA path to the reference's results on machines
where the reference cannot be built. Inputs are stored in the fixtures (not
regenerated from a seed) so they stay valid across numpy versions. Final
folds are stored in full when small and always as a SHA-256 of their bytes.
"""

from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# name -> (nsamps, tsamp, nbins, eta, param_limits, seed)
FFA_CASES = {
    "ffa_freq_nb32": (8192, 64e-6, 32, 1.0, [[50.0, 60.0]], 1),
    "ffa_freq_nb64": (8192, 64e-6, 64, 1.0, [[70.0, 90.0]], 2),
    "ffa_accel_nb16": (16384, 8e-3, 16, 1.0, [[-1000.0, 1000.0], [10.0, 10.3]], 3),
    "ffa_jerk_nb16": (16384, 8e-3, 16, 1.0, [[-100.0, 100.0], [-900.0, 900.0], [10.0, 10.2]], 4),
}
WIDTHS = np.array([1, 2, 3, 4, 6, 8, 12], dtype=np.uint64)
FOLD_KEEP = 1 << 15  # store folds in full up to this many floats


def series(n: int, seed: int) -> tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng(seed)
    ts_e = rng.standard_normal(n).astype(np.float32)
    ts_v = (1.0 + 0.25 * rng.random(n)).astype(np.float32)
    return ts_e, ts_v


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main() -> None:
    if not ref.available():
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` first")
    for name, (nsamps, tsamp, nbins, eta, lims, seed) in FFA_CASES.items():
        ts_e, ts_v = series(nsamps, seed)
        cfg = ref.make_cfg(nsamps, tsamp, nbins, eta, lims)
        ffa = ref.RefFFA(cfg)
        fold = ffa.execute(ts_e, ts_v).copy()
        coords = ref.resolve(cfg, ffa.coord_size)
        widths = WIDTHS[WIDTHS < nbins]
        scores = ref.snr_boxcar_3d(fold, widths, nbins)
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            ts_e=ts_e, ts_v=ts_v, nsamps=nsamps, nbins=nbins, eta=eta, tsamp=tsamp,
            param_limits=np.array(lims, dtype=np.float64),
            n_levels=ffa.n_levels, bseg_brute=ffa.bseg_brute, ncoords=ffa.ncoords,
            param_counts=ffa.param_counts, dparams=ffa.dparams,
            ncoords_offsets=ffa.ncoords_offsets,
            coords=coords.view(np.uint32).reshape(coords.size, -1),
            fold=fold if fold.size <= FOLD_KEEP else fold[:0], fold_sha256=sha(fold),
            fold_size=fold.size, widths=widths, scores=scores,
        )
        print(name, "levels", ffa.n_levels, "final counts", ffa.param_counts[-1].tolist())

    # Brute fold with an explicit frequency list (reference test shape,
    # tests/python/test_cpu_match.py:20-61, scaled down).
    ts_e, ts_v = series(1 << 14, 5)
    freqs = np.linspace(140.0, 145.0, 7)
    bf = ref.brute_fold(ts_e, ts_v, freqs, 1 << 11, 64, 64e-6, 0.0)
    np.savez_compressed(os.path.join(OUT, "brute_fold_nb64.npz"), ts_e=ts_e, ts_v=ts_v, freqs=freqs,
                        segment_len=1 << 11, nbins=64, tsamp=64e-6, t_ref=0.0, fold=bf)

    # Boxcar scores of random (E, V) folds, per width and max; width trials.
    rng = np.random.default_rng(6)
    folds = np.empty((96, 2, 48), dtype=np.float32)
    folds[:, 0] = rng.standard_normal((96, 48)) * 10
    folds[:, 1] = 50 + rng.random((96, 48)) * 10
    widths = np.array([1, 2, 3, 5, 8, 13], dtype=np.uint64)
    np.savez_compressed(os.path.join(OUT, "scores_nb48.npz"), folds=folds, widths=widths,
                        scores=ref.snr_boxcar_3d(folds, widths, 48),
                        scores_max=ref.snr_boxcar_3d_max(folds, widths, 48),
                        trials_64=ref.box_widths(64), trials_128=ref.box_widths(128),
                        trials_100_03=ref.box_widths(100, 0.3, 1.5))

    # Phase-index known answers straight from psr_utils::get_phase_idx[_uint].
    pts = []
    for t, f, nb, d in [(0.0, 10.0, 64, 0.0), (0.1, 10.0, 64, 0.0), (12.3456, 47.3, 128, 0.0),
                        (-0.25, 21.14, 128, 1e-3), (1.0, 1.0, 32, 0.0), (0.49999, 2.0, 64, 0.0),
                        (134.2, 50.0, 128, 0.0), (0.0123, 199.9, 32, -0.004),
                        (0.0078125, 63.99, 64, 0.0), (3.0, 0.333333333333, 16, 0.0)]:
        pts.append((t, f, nb, d, ref.phase_idx(t, f, nb, d), ref.phase_idx_uint(t, f, nb, d)))
    np.savez_compressed(os.path.join(OUT, "phase_idx.npz"), cases=np.array(pts, dtype=np.float64))
    print("done")


# Pruning runs: name -> (nsamps, tsamp, nbins, eta, param_limits, bseg_ffa, seed,
# max_sugg, batch_size, thr_lo, thr_hi, conservative). The small world-tree
# capacities force the overload path (threshold raised by order statistics).
PRUNE_CASES = {
    "prune_accel_nb16": (16384, 8e-3, 16, 1.0, [[-1000.0, 1000.0], [10.0, 10.3]], 2048, 5,
                         64, 8, 1.0, 2.5, False),
    "prune_jerk_nb16": (16384, 8e-3, 16, 1.0, [[-100.0, 100.0], [-900.0, 900.0], [10.0, 10.2]],
                        2048, 6, 64, 8, 1.0, 2.5, True),
}


# The same runs in the Chebyshev basis (poly_basis "chebyshev"; the
# reference rejects the conservative tile there).
CHEBY_CASES = {
    "prune_cheby_accel_nb16": (16384, 8e-3, 16, 1.0, [[-1000.0, 1000.0], [10.0, 10.3]], 2048, 5,
                               64, 8, 1.0, 2.5, False),
    "prune_cheby_jerk_nb16": (16384, 8e-3, 16, 1.0, [[-100.0, 100.0], [-900.0, 900.0], [10.0, 10.2]],
                              2048, 6, 64, 8, 1.0, 2.5, False),
}


def prune_fixtures() -> None:
    """Inputs (the reference's final FFA fold) and outputs of whole pruning
    runs (PruneImpl over the reference's PruneDPFuncts and WorldTree), plus
    branching patterns."""
    cases = [(n, c, "taylor") for n, c in PRUNE_CASES.items()] + [(n, c, "chebyshev") for n, c in CHEBY_CASES.items()]
    for name, (ns, ts, nb, eta, lims, bf, seed, ms, bs, lo, hi, cons), basis in cases:
        cfg = ref.make_cfg(ns, ts, nb, eta, lims, bseg_ffa=bf)
        ffa = ref.RefFFA(cfg)
        ts_e, ts_v = series(ns, seed)
        fold = ffa.execute(ts_e, ts_v).copy()
        nseg = int(ffa.nsegments[-1])
        bp0 = ref.branching_pattern_basis(cfg, basis, 0, cons)
        bmax = max(int(np.ceil(bp0.max() * 2)), 32)
        if basis == "taylor":
            assert bmax == ref.branch_max(cfg, cons)
        thr = np.linspace(lo, hi, nseg - 1).astype(np.float32)
        ref_seg = nseg // 2
        stats, leaves, folds, scores = ref.prune_run(cfg, fold, thr, ref_seg, ms, bs, bmax, nseg - 1, nb, cons,
                                                     basis=basis)
        # whole runs as PruneImpl::run ends them: survivors ascended to the
        # middle of the data and reported there, after every level and after
        # half of them
        fin = ref.prune_run_full(cfg, fold, thr, ref_seg, ms, bs, bmax, nseg - 1, nb, cons, basis=basis)
        half = ref.prune_run_full(cfg, fold, thr, ref_seg, ms, bs, bmax, (nseg - 1) // 2, nb, cons, basis=basis)
        finals = {}
        for tag, (st, lv, fo, sc, ep) in (("final", fin), ("half", half)):
            finals.update({f"{tag}_levels": st.size - 1, f"{tag}_leaves": lv, f"{tag}_folds": fo,
                           f"{tag}_scores": sc, f"{tag}_scores_ep": ep})
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            nsamps=ns, tsamp=ts, nbins=nb, eta=eta, param_limits=np.array(lims, dtype=np.float64),
            bseg_ffa=bf, ffa_fold=fold, thresholds=thr, ref_seg=ref_seg, max_sugg=ms, batch_size=bs,
            branch_max=bmax, conservative=int(cons),
            stats=np.stack([stats[k].astype(np.float64) for k in
                            ("level", "seg_idx", "n_branches", "n_leaves", "n_leaves_phy",
                             "n_leaves_surv", "threshold", "score_min", "score_max")], axis=1),
            leaves=leaves, folds=folds, scores=scores, basis=basis,
            branching_pattern=bp0,
            branching_pattern_ref=ref.branching_pattern_basis(cfg, basis, ref_seg, cons),
            **finals,
        )
        print(name, "nsegments", nseg, "survivors", leaves.shape[0])


# Frequency-sweep chunk plans: name -> (nsamps, tsamp, nbins, eta, param_limits,
# max_process_memory_gb, max_passing_candidates, use_gpu). The small memory
# limits force the bisection, sliver and drift-widening paths.
SWEEP_PLAN_CASES = {
    "accel_2p22_8gb_cpu": (1 << 22, 64e-6, 64, 2.0, [[-200.0, 200.0], [1.0, 500.0]], 8.0, 1 << 22, False),
    "accel_2p22_8gb_gpu": (1 << 22, 64e-6, 64, 2.0, [[-200.0, 200.0], [1.0, 500.0]], 8.0, 1 << 22, True),
    "freq_2p22_2gb_gpu": (1 << 22, 64e-6, 32, 1.0, [[0.5, 800.0]], 2.0, 1 << 22, True),
    "jerk_2p20_3gb_cpu": (1 << 20, 64e-6, 32, 2.0, [[-30.0, 30.0], [-300.0, 300.0], [5.0, 200.0]], 3.0, 1 << 20,
                          False),
    "freq_2p16_tight_gpu": (1 << 16, 1e-3, 32, 1.0, [[1.0, 40.0]], 0.508, 4096, True),
    "freq_2p16_tight_cpu": (1 << 16, 1e-3, 32, 1.0, [[1.0, 40.0]], 0.508, 4096, False),
    "accel_2p16_tight_gpu": (1 << 16, 1e-3, 32, 2.0, [[-50.0, 50.0], [2.0, 30.0]], 0.503, 4096, True),
    "jerk_2p15_tight_gpu": (1 << 15, 2e-3, 16, 2.0, [[-2.0, 2.0], [-20.0, 20.0], [2.0, 12.0]], 0.5004, 4096,
                            True),
}

# Whole sweeps (reference planner + reference FFA and scores per chunk +
# compaction + save_results decode): name -> (plan case, snr_min, seed,
# pulsars (f0, amplitude, duty)).
SWEEP_RUN_CASES = {
    "sweep_freq_2p16": ("freq_2p16_tight_gpu", 6.0, 21, [(3.3, 0.6, 0.05), (17.9, 0.5, 0.03)]),
    "sweep_accel_2p16": ("accel_2p16_tight_gpu", 6.0, 22, [(5.1, 0.5, 0.05), (24.4, 0.5, 0.04)]),
    "sweep_jerk_2p15": ("jerk_2p15_tight_gpu", 4.5, 23, [(7.7, 0.6, 0.05), (3.2, 0.5, 0.05)]),
}


def _ref_backend(nsamps, tsamp, nbins, eta, lims, ts_e, ts_v, widths=None):
    cfg = ref.make_cfg(nsamps, tsamp, nbins, eta, lims)
    ffa = ref.RefFFA(cfg)
    w = ref.box_widths(nbins) if widths is None else np.asarray(widths, np.uint64)
    fold = ffa.execute(ts_e, ts_v).copy()
    return ref.snr_boxcar_3d(fold, w, nbins).ravel(), ffa.param_counts[-1].copy(), w


def sweep_fixtures() -> None:
    from oracle import sweep as osweep

    plans = {}
    for name, (nsamps, tsamp, nbins, eta, lims, mem, mp, gpu) in SWEEP_PLAN_CASES.items():
        rows, stats = ref.region_plan(ref.make_cfg(nsamps, tsamp, nbins, eta, lims), mem, 2.0, 1024, mp, gpu)
        plans[f"{name}__rows"] = rows
        plans[f"{name}__stats"] = stats
        plans[f"{name}__inputs"] = np.array([nsamps, tsamp, nbins, eta, mem, mp, float(gpu)], np.float64)
        plans[f"{name}__lims"] = np.array(lims, np.float64)
        print(name, "chunks", rows.shape[0])
    np.savez_compressed(os.path.join(OUT, "sweep_plans.npz"), **plans)

    for name, (pcase, snr_min, seed, psrs) in SWEEP_RUN_CASES.items():
        nsamps, tsamp, nbins, eta, lims, mem, mp, gpu = SWEEP_PLAN_CASES[pcase]
        ts_e, ts_v = series(nsamps, seed)
        t = np.arange(nsamps) * tsamp
        for f0, amp, duty in psrs:
            ts_e += (amp * (np.mod(t * f0, 1.0) < duty)).astype(np.float32)
        rows, _ = ref.region_plan(ref.make_cfg(nsamps, tsamp, nbins, eta, lims), mem, 2.0, 1024, mp, gpu)
        base = (nsamps, tsamp, nbins, eta, lims)
        out = {}
        for tag, chunk_w in (("base_widths", False), ("chunk_widths", True)):
            params, snr, counts = osweep.run(base, rows[:, :4], ts_e, ts_v, snr_min, backend=_ref_backend,
                                             chunk_widths=chunk_w)
            out[f"params_{tag}"] = params
            out[f"snr_{tag}"] = snr
            out["region_counts"] = counts
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), ts_e=ts_e, ts_v=ts_v, nsamps=nsamps, tsamp=tsamp,
                            nbins=nbins, eta=eta, param_limits=np.array(lims, np.float64), max_memory_gb=mem,
                            max_passing=mp, snr_min=snr_min, chunks=rows, **out)
        print(name, "chunks", rows.shape[0], "candidates", out["snr_base_widths"].size,
              out["region_counts"].tolist())


# name -> (nstages, branching (lo, hi), ref_ducy, keyword arguments of the scheme)
DTS_CASES = {
    "dts_nb32": (8, (1.5, 4.0), 0.1, dict(nbins=32, ntrials=256, nprobs=6, nthresholds=50, thres_neigh=6)),
    "dts_nb48": (10, (1.5, 4.0), 0.1, dict(nbins=48, ntrials=128, nprobs=8, nthresholds=60, thres_neigh=10,
                                           ducy_max=0.2, wtsp=1.5, snr_final=7.0)),
}


def dts_fixtures() -> None:
    """DynamicThresholdScheme: the reference's set-up pieces and the stage
    loop restated over them (ref_capi.cpp), with the oracle's guess path (the
    reference's norm_isf needs Boost.Math) and normal quantile table."""
    from oracle import lko

    lut = lko.dts_normal_lut()
    for name, (ns, (lo, hi), ducy, kw) in DTS_CASES.items():
        bp = np.linspace(lo, hi, ns).astype(np.float32)
        snr_final = kw.get("snr_final", 8.0)
        guess = lko.dts_guess(ns, snr_final, bp)
        states = ref.dts_run(bp, ducy, guess, lut, lko.DTS_STATE_DTYPE, **kw)
        nthr, nprobs = kw["nthresholds"], kw["nprobs"]
        thr = ref.dts_thresholds(0.1, snr_final, nthr)
        probs = ref.dts_probs(nprobs, kw.get("prob_min", 0.05))
        best = ref.dts_best_path(states, ns, thr, probs, 0.1)
        fields = {f"state_{f}": states[f] for f in lko.DTS_STATE_DTYPE.names if f != "_pad"}
        np.savez_compressed(os.path.join(OUT, f"{name}.npz"), branching=bp, ref_ducy=ducy, guess=guess,
                            lut_sha256=sha(lut), thresholds=thr, probs=probs,
                            profile=ref.dts_profile(kw["nbins"], ducy), bound=ref.dts_bound(ns, snr_final),
                            best_path=best, config=np.array([repr(kw)]), **fields)
        print(name, "non-empty states", int((~states["is_empty"]).sum()), "best path", best.tolist())


# Fourier-domain FFA (FFA<ComplexType>): name -> (nsamps, tsamp, nbins, eta,
# param_limits, seed). nbins 128 takes the lossy level 0 (time-domain brute
# fold + real transform); the reference's FFTW calls run through the
# DFT-definition stand-in of oracle/ref_stubs.cpp.
FOURIER_CASES = {
    "fourier_freq_nb32": (16384, 64e-6, 32, 1.0, [[50.0, 60.0]], 21),
    "fourier_freq_nb64": (8192, 64e-6, 64, 1.0, [[70.0, 90.0]], 22),
    "fourier_accel_nb16": (16384, 8e-3, 16, 1.0, [[-1000.0, 1000.0], [10.0, 10.3]], 23),
    "fourier_jerk_nb16": (16384, 8e-3, 16, 1.0, [[-100.0, 100.0], [-900.0, 900.0], [10.0, 10.2]], 24),
    "fourier_freq_nb128_lossy": (8192, 64e-6, 128, 1.0, [[70.0, 90.0]], 25),
}


def fourier_fixtures() -> None:
    for name, (nsamps, tsamp, nbins, eta, lims, seed) in FOURIER_CASES.items():
        ts_e, ts_v = series(nsamps, seed)
        cfg = ref.make_cfg(nsamps, tsamp, nbins, eta, lims)
        ffa = ref.RefFourier(cfg)
        fold = ffa.execute(ts_e, ts_v).copy()
        fold_time = ffa.execute_time(ts_e, ts_v).copy()
        plan = ref.RefFFA(cfg)
        nw = ref.box_widths(nbins).size
        scores = ref.fourier_scores(cfg, ts_e, ts_v, int(plan.ncoords[-1]) * nw)
        np.savez_compressed(
            os.path.join(OUT, f"{name}.npz"),
            ts_e=ts_e, ts_v=ts_v, nsamps=nsamps, nbins=nbins, eta=eta, tsamp=tsamp,
            param_limits=np.array(lims, dtype=np.float64), n_levels=plan.n_levels,
            ncoords=plan.ncoords, fold=fold if fold.size <= FOLD_KEEP else fold[:0],
            fold_size=fold.size, fold_time=fold_time if fold_time.size <= FOLD_KEEP else fold_time[:0],
            scores=scores, widths=ref.box_widths(nbins),
        )
        print(name, "levels", plan.n_levels, "final coords", int(plan.ncoords[-1]), "fold", fold.size)

    # Direct transform with an explicit frequency list (reference test shape,
    # tests/python/test_cpu_match.py:20-61, scaled down), odd nbins included.
    ts_e, ts_v = series(1 << 14, 26)
    freqs = np.linspace(140.0, 145.0, 7)
    out = {}
    for nb in (64, 33):
        out[f"fold_nb{nb}"] = ref.brute_fold_complex(ts_e, ts_v, freqs, 1 << 11, nb, 64e-6, 0.0123)
    np.savez_compressed(os.path.join(OUT, "brute_fold_fourier.npz"), ts_e=ts_e, ts_v=ts_v, freqs=freqs,
                        segment_len=1 << 11, tsamp=64e-6, t_ref=0.0123, **out)
    print("brute_fold_fourier", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if not ref.available():
        raise SystemExit("oracle/_ref is not built: run `make -C oracle ref` first")
    if len(sys.argv) > 1 and sys.argv[1] == "prune":
        prune_fixtures()
    elif len(sys.argv) > 1 and sys.argv[1] == "sweep":
        sweep_fixtures()
    elif len(sys.argv) > 1 and sys.argv[1] == "dts":
        dts_fixtures()
    elif len(sys.argv) > 1 and sys.argv[1] == "fourier":
        fourier_fixtures()
    else:
        main()
        prune_fixtures()
        sweep_fixtures()
        dts_fixtures()
        fourier_fixtures()
