"""Pruning tree on the GPU: ``PruneCUDA`` (one run for one reference segment)
and ``EPMultiPassCUDA`` (FFA to ``bseg_ffa`` segments, then one pruning run per
reference segment), mirroring ``libloki.prune.EPMultiPassTime`` of the
reference (src/loki_templates.hpp:87-113, lib/prune.cpp:626-930).

Each run seeds the world tree from the final FFA level of the reference
segment and prunes level by level in middle-out segment order with the
reference's batch, threshold and world-tree semantics (branch, resolve,
shift-add, max-width boxcar S/N, filter ``score >= threshold``, transform,
add with overload pruning). Results match the reference's CPU code bit for
bit. The ascend / report stage and the HDF5 writer are not part of this
module: runs return the final tree (leaves, folds, scores) and the per-level
statistics, and ``execute`` can save them as ``.npz`` plus a text log.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _capi as C
from . import _device as D
from .configs import PulsarSearchConfig
from .ffa import FFACUDA

PRUNE_STATS_DTYPE = np.dtype([
    ("level", np.uint64), ("seg_idx", np.uint64), ("n_branches", np.uint64), ("n_leaves", np.uint64),
    ("n_leaves_phy", np.uint64), ("n_leaves_surv", np.uint64), ("threshold", np.float32),
    ("score_min", np.float32), ("score_max", np.float32), ("pad", np.float32)])


_BASES = {"taylor": 0, "chebyshev": 1}


def _basis(poly_basis: str) -> int:
    if poly_basis not in _BASES:
        raise ValueError(f"Unknown poly_basis: '{poly_basis}'. Valid options: 'taylor', 'chebyshev'")
    return _BASES[poly_basis]


def branching_pattern(cfg: PulsarSearchConfig, ref_seg: int = 0, use_conservative_tile: bool = False,
                      poly_basis: str = "taylor") -> np.ndarray:
    """FFAPlan.get_branching_pattern(poly_basis, ref_seg): generate_bp_poly_taylor
    (lib/taylor.cpp:1643-1741) or generate_bp_poly_chebyshev (lib/chebyshev.cpp:1796-1890)."""
    b = _basis(poly_basis)
    out = np.zeros(4096, np.float64)
    n = ctypes.c_uint64()
    C.check(C.lib().lk_plan_branching_pattern_basis(cfg._plan_handle, int(ref_seg), int(use_conservative_tile), b,
                                                    out.ctypes.data, out.size, ctypes.byref(n)))
    if n.value > out.size:
        out = np.zeros(n.value, np.float64)
        C.check(C.lib().lk_plan_branching_pattern_basis(cfg._plan_handle, int(ref_seg), int(use_conservative_tile),
                                                        b, out.ctypes.data, out.size, ctypes.byref(n)))
    return out[: n.value].copy()


def middle_out_order(nsegments: int, ref_seg: int) -> list[int]:
    """MiddleOutScheme's segment order (lib/loki/psr_utils.hpp:331-347):
    stable argsort of |i - ref_seg|."""
    return sorted(range(nsegments), key=lambda i: (abs(i - ref_seg), i))


def determine_ref_segs(nsegments: int, n_runs: int | None = None, ref_segs=None) -> list[int]:
    """utils::determine_ref_segs_pareto (lib/utils.cpp:243-278)."""
    if n_runs is not None:
        if n_runs < 1 or n_runs > nsegments:
            raise RuntimeError(f"n_runs must be between 1 and {nsegments}, got {n_runs}")
        if n_runs == 1:
            return [nsegments // 2]

        def round_div(num, den):
            return (num + den // 2) // den

        margin = round_div(nsegments - 1, 2 * n_runs)
        lo, hi, denom = margin, nsegments - 1 - margin, n_runs - 1
        return [round_div((denom - i) * lo + i * hi, denom) for i in range(n_runs)]
    if ref_segs is not None:
        return [int(r) for r in ref_segs]
    raise RuntimeError("Either n_runs or ref_segs must be provided")


class PruneCUDA:
    """One pruning search over the final FFA level of ``cfg`` on one device.

    ``max_sugg`` is the world-tree capacity, ``batch_size`` the parents per
    batch (it decides when overload pruning raises the threshold, exactly as
    in the reference), ``branch_max`` the most child values of one parameter
    (None: EPMultiPass's rule, max(ceil(2 * max branching), 32)) and
    ``poly_basis`` "taylor" or "chebyshev" (lib/dynamic.cpp:381-450).
    """

    def __init__(self, cfg: PulsarSearchConfig, max_sugg: int = 1 << 20, batch_size: int = 4096,
                 branch_max: int | None = None, use_conservative_tile: bool = False, device_id: int = 0,
                 poly_basis: str = "taylor"):
        D.require_cuda(device_id)
        if cfg.nparams not in (2, 3):
            raise NotImplementedError("pruning is implemented for searches with nparams 2 or 3")
        self.poly_basis = poly_basis
        basis = _basis(poly_basis)
        self._cfg = cfg
        self._device = device_id
        self._nparams = cfg.nparams
        self._nbins = cfg.nbins
        h = ctypes.c_void_p()
        with D.torch().cuda.device(device_id):
            C.check(C.lib().lk_prune_create_basis(cfg._plan_handle, int(max_sugg), int(batch_size),
                                                  0 if branch_max is None else int(branch_max),
                                                  int(use_conservative_tile), basis, device_id, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                C.lib().lk_prune_destroy(h)
            except Exception:
                pass
            self._h = None

    def set_persistent_tail(self, enable: bool = True) -> None:
        """Run the levels of a small tree in one persistent cooperative launch
        (the default) or level by level with host round trips; results are
        identical."""
        C.check(C.lib().lk_prune_set_tail(self._h, int(bool(enable))))

    def run(self, ffa_fold, ref_seg: int, thresholds, n_iters: int | None = None) -> np.ndarray:
        """Seed from segment ``ref_seg`` of the final FFA fold (CUDA tensor or host
        array, [nsegments, ncoords, 2, nbins]) and prune; returns the per-level
        statistics (one row for the seed, then one per level run)."""
        fold = D.to_device_f32(ffa_fold, self._device).reshape(-1)
        thr = np.ascontiguousarray(thresholds, dtype=np.float32)
        n_iters = thr.size if n_iters is None else int(n_iters)
        stats = (C.LkPruneStats * (n_iters + 1))()
        n = ctypes.c_uint64()
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_prune_run(self._h, D.ptr(fold), int(ref_seg), thr.ctypes.data, thr.size, n_iters,
                                         stats, n_iters + 1, ctypes.byref(n), D.stream_ptr(self._device)))
        out = np.zeros(n.value, PRUNE_STATS_DTYPE)
        for i in range(n.value):
            for name in PRUNE_STATS_DTYPE.names:
                out[name][i] = getattr(stats[i], name)
        return out

    @staticmethod
    def run_many(prunes, ffa_fold, ref_segs, thresholds, n_iters: int | None = None) -> list:
        """One run per executor (``prunes[k]`` seeds from ``ref_segs[k]``; same
        configuration, distinct executors, one device) on the current stream:
        each run's large levels level by level, then the small trees' tails of
        all runs in ONE cooperative launch. Returns each run's statistics, as
        ``run`` gives them; each executor then holds its run's tree."""
        prunes = list(prunes)
        if len(prunes) != len(ref_segs) or not prunes:
            raise ValueError("one executor per reference segment")
        dev = prunes[0]._device
        fold = D.to_device_f32(ffa_fold, dev).reshape(-1)
        thr = np.ascontiguousarray(thresholds, dtype=np.float32)
        n_iters = thr.size if n_iters is None else int(n_iters)
        k = len(prunes)
        per = n_iters + 1
        stats = (C.LkPruneStats * (k * per))()
        counts = (ctypes.c_uint64 * k)()
        handles = (ctypes.c_void_p * k)(*[p._h.value for p in prunes])
        segs = np.ascontiguousarray(ref_segs, dtype=np.uint64)
        with D.torch().cuda.device(dev):
            C.check(C.lib().lk_prune_run_many(handles, k, D.ptr(fold), segs.ctypes.data, thr.ctypes.data, thr.size,
                                              n_iters, stats, per, counts, D.stream_ptr(dev)))
        out = []
        for j in range(k):
            rows = np.zeros(counts[j], PRUNE_STATS_DTYPE)
            for i in range(counts[j]):
                for name in PRUNE_STATS_DTYPE.names:
                    rows[name][i] = getattr(stats[j * per + i], name)
            out.append(rows)
        return out

    def finalize(self, ffa_fold) -> None:
        """Ascend the run's survivors to the middle of the data and report them
        there (the end of the reference's PruneImpl::run): folds over every
        segment searched, their scores, the run's scores kept as scores_ep,
        leaves as observer-frame Taylor parameters."""
        fold = D.to_device_f32(ffa_fold, self._device).reshape(-1)
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_prune_finalize(self._h, D.ptr(fold), D.stream_ptr(self._device)))

    def scores_ep(self, host: bool = True):
        """scores_ep of the finalized tree, logical order."""
        t = D.torch()
        n = self.tree_size
        out = t.empty(max(n, 1), dtype=t.float32, device=f"cuda:{self._device}")
        with t.cuda.device(self._device):
            C.check(C.lib().lk_prune_get_scores_ep(self._h, out.data_ptr(), max(n, 1),
                                                   D.stream_ptr(self._device)))
        out = out[:n]
        return out.cpu().numpy() if host else out

    @property
    def tree_size(self) -> int:
        n = ctypes.c_uint64()
        C.check(C.lib().lk_prune_tree_size(self._h, ctypes.byref(n)))
        return n.value

    def tree(self, host: bool = True):
        """Final tree in logical order: (leaves [n, nparams+2, 2] f64, folds
        [n, 2, nbins] f32, scores [n] f32), as host arrays or CUDA tensors."""
        t = D.torch()
        n = self.tree_size
        dev = f"cuda:{self._device}"
        leaves = t.empty((max(n, 1), self._nparams + 2, 2), dtype=t.float64, device=dev)
        folds = t.empty((max(n, 1), 2, self._nbins), dtype=t.float32, device=dev)
        scores = t.empty(max(n, 1), dtype=t.float32, device=dev)
        with t.cuda.device(self._device):
            C.check(C.lib().lk_prune_get_tree(self._h, leaves.data_ptr(), folds.data_ptr(), scores.data_ptr(),
                                              max(n, 1), D.stream_ptr(self._device)))
        leaves, folds, scores = leaves[:n], folds[:n], scores[:n]
        if host:
            return leaves.cpu().numpy(), folds.cpu().numpy(), scores.cpu().numpy()
        return leaves, folds, scores


class EPMultiPassCUDA:
    """FFA to ``bseg_ffa`` segments, then one pruning run per reference segment
    (reference ``EPMultiPass``: same arguments; ``device_id`` added).

    ``n_workers`` (default ``cfg.nthreads``, the reference's number of pruning
    workspaces) runs that many reference segments at once on the device (the
    reference runs its segments on a thread pool of ``nthreads``
    workspaces). ``batched=True`` (default): each group of ``n_workers`` runs
    goes through ``PruneCUDA.run_many`` on one stream, the small trees' tails
    of the group in one cooperative launch; ``batched=False``: each worker on
    its own executor, CUDA stream and host thread. Results do not depend on
    either. Each worker
    takes a fixed share of the segments (its executor's buffers then stop
    growing after the first execute). No more workers run than there are
    reference segments to prune, and each worker's executor (device buffers
    sized for ``max_sugg`` leaves) is created when the worker first runs.
    Eight segments of the jerk search (FFA included): 17.9 ms one at a time,
    8.9 ms batched (9.9 ms on eight threads and streams)."""

    def __init__(self, cfg: PulsarSearchConfig, threshold_scheme, n_runs: int | None = None, ref_segs=None,
                 max_sugg: int = 1 << 18, batch_size: int = 1024, poly_basis: str = "taylor",
                 show_progress: bool = False, use_conservative_tile: bool = False, device_id: int = 0,
                 n_workers: int | None = None, batched: bool = True):
        _basis(poly_basis)
        self._cfg = cfg
        self._thr = np.ascontiguousarray(threshold_scheme, dtype=np.float32)
        self._n_runs = n_runs
        self._ref_segs = ref_segs
        self._ffa = FFACUDA(cfg, device_id)
        # the reference runs its segments on cfg.nthreads workspaces
        self._workers = max(1, int(cfg.nthreads if n_workers is None else n_workers))
        self._prune_args = (cfg, max_sugg, batch_size, None, use_conservative_tile, device_id)
        self._poly_basis = poly_basis
        self._prunes: list[PruneCUDA] = []
        self._device = device_id
        self._batched = bool(batched)

    def _executor(self, k: int) -> "PruneCUDA":
        """Worker k's pruning executor, created on first use."""
        while len(self._prunes) <= k:
            self._prunes.append(PruneCUDA(*self._prune_args, poly_basis=self._poly_basis))
        return self._prunes[k]

    def _result(self, pr: "PruneCUDA", fold, ref_seg: int, nseg: int, stats) -> dict:
        pr.finalize(fold)
        leaves, folds, scores = pr.tree()
        return {"stats": stats, "leaves": leaves, "folds": folds, "scores": scores,
                "scores_ep": pr.scores_ep(),
                "snail_scheme": np.array(middle_out_order(nseg, ref_seg), np.uint64)}

    def _run_one(self, pr: "PruneCUDA", fold, ref_seg: int, nseg: int, stream) -> dict:
        t = D.torch()
        with t.cuda.device(self._device), t.cuda.stream(stream):
            stats = pr.run(fold, ref_seg, self._thr, n_iters=nseg - 1)
            return self._result(pr, fold, ref_seg, nseg, stats)

    @property
    def ffa(self) -> FFACUDA:
        return self._ffa

    def execute(self, ts_e, ts_v, outdir: str | None = None, file_prefix: str = "test") -> dict:
        """Runs every reference segment as the reference's PruneImpl::run does
        (levels, then survivors ascended and reported at the middle of the
        data). Returns {ref_seg: {"stats", "leaves", "folds", "scores",
        "scores_ep", "snail_scheme"}}; with ``outdir`` also writes
        ``<prefix>_pruning_nstages_<n>_results.npz`` (per run ``<ref_seg>_00``:
        param_sets, scores, scores_ep, snail_scheme, level_stats -- the
        reference's HDF5 run group) and a text log."""
        t = D.torch()
        fold = self._ffa.execute(D.to_device_f32(ts_e, self._device), D.to_device_f32(ts_v, self._device))
        nseg = int(self._ffa.plan.nsegments[-1])
        segs = determine_ref_segs(nseg, self._n_runs, self._ref_segs)
        t.cuda.synchronize(self._device)  # the fold is complete before other streams read it
        workers = max(1, min(self._workers, len(segs)))
        if self._batched and workers > 1:
            # groups of `workers` runs, each group's tails in one launch
            prunes = [self._executor(k) for k in range(workers)]
            runs = []
            with t.cuda.device(self._device):
                for g0 in range(0, len(segs), workers):
                    group = segs[g0 : g0 + workers]
                    stats = PruneCUDA.run_many(prunes[: len(group)], fold, group, self._thr, n_iters=nseg - 1)
                    runs += [self._result(pr, fold, rs, nseg, st) for pr, rs, st in zip(prunes, group, stats)]
        elif workers == 1:
            stream = t.cuda.current_stream(self._device)
            pr = self._executor(0)
            runs = [self._run_one(pr, fold, rs, nseg, stream) for rs in segs]
        else:
            from concurrent.futures import ThreadPoolExecutor

            prunes = [self._executor(k) for k in range(workers)]
            streams = [t.cuda.Stream(device=self._device) for _ in range(workers)]
            # A fixed share of the segments per worker: each executor sees the
            # same runs on every execute, so its buffers stop growing after the
            # first (a growth frees device memory, which waits for the device).
            shares = [segs[k::workers] for k in range(workers)]

            def work(k):
                return [self._run_one(prunes[k], fold, rs, nseg, streams[k]) for rs in shares[k]]

            with ThreadPoolExecutor(workers) as pool:
                done = list(pool.map(work, range(workers)))
            by_seg = {rs: r for k in range(workers) for rs, r in zip(shares[k], done[k])}
            runs = [by_seg[rs] for rs in segs]
        results = dict(zip(segs, runs))
        if outdir is not None:
            os.makedirs(outdir, exist_ok=True)
            base = os.path.join(outdir, f"{file_prefix}_pruning_nstages_{nseg}")
            arrays = {}
            with open(base + "_log.txt", "w") as log:
                log.write("Pruning log\n")
                for rs, r in results.items():
                    log.write(f"Pruning log for ref segment: {rs}\n")
                    for row in r["stats"]:
                        log.write(f"level {int(row['level'])} seg {int(row['seg_idx'])} thr {row['threshold']:.3f} "
                                  f"branches {int(row['n_branches'])} leaves {int(row['n_leaves'])} "
                                  f"survivors {int(row['n_leaves_surv'])} "
                                  f"score [{row['score_min']:.3f}, {row['score_max']:.3f}]\n")
                    run = f"{rs:03d}_00"
                    arrays[f"{run}/param_sets"] = r["leaves"]
                    arrays[f"{run}/scores"] = r["scores"]
                    arrays[f"{run}/scores_ep"] = r["scores_ep"]
                    arrays[f"{run}/snail_scheme"] = r["snail_scheme"]
                    arrays[f"{run}/level_stats"] = r["stats"]
            np.savez(base + "_results.npz", **arrays)
        return results
