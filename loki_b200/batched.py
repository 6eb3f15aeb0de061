"""Searching many time series of uneven length on one GPU.

Each series is padded to the next power of two with ``ts_e = ts_v = 0`` (the
reference requires power-of-two ``nsamps``, lib/configs.cpp:264; padded
samples add nothing to any fold, and the brute fold skips the segments that
hold only padding, in groups of 8), series of one padded length share one
executor (one plan), and are folded, scored and compacted ``max_batch`` at a
time: one launch per level for the whole batch (a batch of series is, level by
level, one series with ``max_batch`` times the segments). Each full batch step
is captured once in a CUDA graph and replayed for every further batch of that
length; a partial last batch runs eagerly.

Each padded length has ``n_slots`` such executors, each on its own stream;
consecutive batches alternate between them, so one batch's brute fold runs
beside the previous batch's merges and scoring, and a batch's candidates are
read back while the next batch computes. The memory budget is split between
the slots; with batches of many series one slot already fills the GPU (the
512-series benchmark measured 7.48 s per step with one slot, 7.55 s with
two), so one slot is the default.

This is the driver of the reference's batched use (``FFAFreqSweep`` over many
beams / DM trials): per series it returns the candidates ``score >= snr_min``
in flat ``coord * n_widths + width`` order, exactly the single-series result.
"""

from __future__ import annotations

import numpy as np

from . import _device as D
from .configs import PulsarSearchConfig
from .ffa import FFACUDA


def _pow2_ceil(n: int) -> int:
    return 1 << max(0, int(n - 1).bit_length())


class _Group:
    """Executor, static buffers and captured graph for one padded length."""

    def __init__(self, cfg: PulsarSearchConfig, nbatch: int, device: int, use_graph: bool, cap: int,
                 fold_storage: str = "fp32"):
        t = D.torch()
        dev = f"cuda:{device}"
        self.cfg = cfg
        self.nbatch = nbatch
        self.ffa = FFACUDA(cfg, device_id=device, max_batch=nbatch, fold_storage=fold_storage)
        self.per = int(self.ffa.plan.ncoords[-1]) * cfg.n_scoring_widths
        n = cfg.nsamps
        self.e = t.zeros((nbatch, n), dtype=t.float32, device=dev)
        self.v = t.zeros((nbatch, n), dtype=t.float32, device=dev)
        self.idx = t.empty(cap, dtype=t.int32, device=dev)
        self.snr = t.empty(cap, dtype=t.float32, device=dev)
        self.cnt = t.zeros(1, dtype=t.int64, device=dev)
        # valid samples of each series of the batch: the brute fold skips the
        # segments that hold only padding (read by the captured graph too)
        self.lens = t.zeros(nbatch, dtype=t.int64, device=dev)
        self.hlens = t.zeros(nbatch, dtype=t.int64).pin_memory()
        self.ffa.set_batch_lengths(self.lens)
        self.use_graph = use_graph
        self.graph = None
        self.stream = t.cuda.Stream(device=dev)
        self.hcnt = t.zeros(1, dtype=t.int64).pin_memory()
        self.done = t.cuda.Event()
        self.pending = None  # (chunk, L) of the batch in flight

    def run(self, nb: int, snr_min: float):
        t = D.torch()
        if nb == self.nbatch and self.use_graph:
            if self.graph is None:
                # warm-up outside capture: every allocation happens here
                self.ffa.search_batch(self.e, self.v, snr_min, self.idx, self.snr, self.cnt)
                t.cuda.synchronize()
                g = t.cuda.CUDAGraph()
                with t.cuda.graph(g):
                    self.ffa.search_batch(self.e, self.v, snr_min, self.idx, self.snr, self.cnt)
                self.graph = g
            self.graph.replay()
        else:
            self.ffa.search_batch(self.e[:nb], self.v[:nb], snr_min, self.idx, self.snr, self.cnt)


class MultiSeriesSearch:
    """FFA period search of many series (``tsamp``, ``nbins``, frequency range
    ``f_range``, boxcar ``widths``, threshold ``snr_min``) on one device.
    ``fold_storage="bf16"`` stores the intermediate levels in BF16 and
    rescores near-threshold cells exactly (same candidates as FP32)."""

    def __init__(self, tsamp: float, nbins: int, f_range, widths, snr_min: float, max_batch: int = 8,
                 eta: float = 1.0, device_id: int = 0, use_graphs: bool = True, max_cands: int = 1 << 22,
                 mem_fraction: float = 0.25, fold_storage: str = "fp32", n_slots: int = 1,
                 autotune: bool = False):
        self.fold_storage = fold_storage
        D.require_cuda(device_id)
        self.tsamp, self.nbins, self.eta = float(tsamp), int(nbins), float(eta)
        self.f_range = (float(f_range[0]), float(f_range[1]))
        self.widths = [int(w) for w in widths]
        self.snr_min = float(snr_min)
        self.max_batch = int(max_batch)
        self.device = device_id
        self.use_graphs = use_graphs
        self.max_cands = int(max_cands)
        self.mem_fraction = float(mem_fraction)
        self.n_slots = max(1, int(n_slots))
        self.autotune = bool(autotune)
        self._tuned: set[int] = set()
        self.groups: dict[int, list[_Group]] = {}

    def config(self, nsamps: int) -> PulsarSearchConfig:
        return PulsarSearchConfig(nsamps, self.tsamp, self.nbins, self.eta, np.array([self.f_range]),
                                  use_fourier=False, score_widths=self.widths, snr_min=self.snr_min)

    def _group(self, L: int) -> list[_Group]:
        if L not in self.groups:
            cfg = self.config(L)
            probe = FFACUDA(cfg, device_id=self.device, max_batch=1, fold_storage=self.fold_storage)
            per_series = probe.workspace_bytes + 8 * L + 4 * int(probe.plan.ncoords[-1]) * cfg.n_scoring_widths
            if self.fold_storage == "bf16":
                # per-cell best S/N, cell list and its values
                per_series += 12 * int(probe.plan.ncoords[-1])
            del probe
            free, _ = D.torch().cuda.mem_get_info(self.device)
            budget = self.mem_fraction * free / self.n_slots
            nb = int(max(1, min(self.max_batch, budget // max(per_series, 1))))
            self.groups[L] = [_Group(cfg, nb, self.device, self.use_graphs, self.max_cands, self.fold_storage)
                              for _ in range(self.n_slots)]
        return self.groups[L]

    def _tune(self, slots: list, L: int, e, v) -> None:
        """Launch shapes timed on the first series of a length (results are
        unchanged), applied to every slot of that length before any capture."""
        if not self.autotune or L in self._tuned:
            return
        t = D.torch()
        e1 = t.zeros(L, dtype=t.float32, device=f"cuda:{self.device}")
        v1 = t.zeros(L, dtype=t.float32, device=f"cuda:{self.device}")
        e1[: e.shape[-1]].copy_(e if isinstance(e, t.Tensor) else t.from_numpy(np.ascontiguousarray(e, np.float32)))
        v1[: v.shape[-1]].copy_(v if isinstance(v, t.Tensor) else t.from_numpy(np.ascontiguousarray(v, np.float32)))
        tuning = slots[0].ffa.autotune(e1, v1, reps=3)
        for g in slots:
            g.ffa.set_tuning(tuning)
        self._tuned.add(L)

    @staticmethod
    def _collect(g: _Group, out: list) -> None:
        if g.pending is None:
            return
        chunk, L = g.pending
        g.pending = None
        g.done.synchronize()
        total = int(g.hcnt.item())
        k_n = min(total, g.idx.numel())
        t = D.torch()
        with t.cuda.stream(g.stream):
            idx = g.idx[:k_n].cpu().numpy().view(np.uint32)
            snr = g.snr[:k_n].cpu().numpy()
        series_of = idx // g.per
        for j, k in enumerate(chunk):
            sel = series_of == j
            out[k] = {"idx": (idx[sel] - j * g.per).astype(np.uint32), "snr": snr[sel],
                      "total": int(sel.sum()), "nsamps": L}

    def search(self, data) -> list[dict]:
        """``data``: sequence of (ts_e, ts_v) host arrays or CUDA tensors.
        Returns, per series in input order, {"idx": uint32 flat indices,
        "snr": float32, "total": number passing, "nsamps": padded length}."""
        t = D.torch()
        order: dict[int, list[int]] = {}
        for k, (e, _) in enumerate(data):
            order.setdefault(_pow2_ceil(int(e.shape[-1])), []).append(k)
        out: list[dict] = [None] * len(data)  # type: ignore[list-item]
        # inputs already queued on the caller's stream are complete before the
        # slot streams read them
        t.cuda.current_stream(self.device).synchronize()
        for L in sorted(order):
            slots = self._group(L)
            ks = order[L]
            self._tune(slots, L, *data[ks[0]])
            nbatch = slots[0].nbatch
            for bi, b0 in enumerate(range(0, len(ks), nbatch)):
                g = slots[bi % len(slots)]
                self._collect(g, out)  # the slot's previous batch
                chunk = ks[b0 : b0 + nbatch]
                with t.cuda.stream(g.stream):
                    # the slot's previous batch has finished (collected above),
                    # so its copy of the lengths has been read
                    g.hlens.zero_()
                    for j, k in enumerate(chunk):
                        g.hlens[j] = int(data[k][0].shape[-1])
                    g.lens.copy_(g.hlens, non_blocking=True)
                    for j, k in enumerate(chunk):
                        e, v = data[k]
                        n = int(e.shape[-1])
                        src_e = e if isinstance(e, t.Tensor) else t.from_numpy(np.ascontiguousarray(e, np.float32))
                        src_v = v if isinstance(v, t.Tensor) else t.from_numpy(np.ascontiguousarray(v, np.float32))
                        g.e[j, :n].copy_(src_e, non_blocking=True)
                        g.v[j, :n].copy_(src_v, non_blocking=True)
                        if n < L:
                            g.e[j, n:].zero_()
                            g.v[j, n:].zero_()
                    g.run(len(chunk), self.snr_min)
                    g.hcnt.copy_(g.cnt, non_blocking=True)
                    g.done.record(g.stream)
                g.pending = (chunk, L)
            for g in slots:
                self._collect(g, out)
        # the caller's stream orders after every slot's work
        cur = t.cuda.current_stream(self.device)
        for L in order:
            for g in self.groups[L]:
                cur.wait_stream(g.stream)
        return out
