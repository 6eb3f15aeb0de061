"""Host-to-device search pipeline for a stream of series.

``SearchPipeline(ffa, snr_min).run(series)`` searches every (ts_e, ts_v) host
pair of an iterable with the executor ``ffa`` and yields, per series and in
order, the candidates ``score >= snr_min`` (flat ``coord * n_widths + width``
indices, S/N, total) -- what ``FFACUDA.search`` returns for one series. The
copies overlap the searches: while series k is searched, series k + 1 is
copied to the device on a copy stream, and series k - 1's candidates are read
back through pinned buffers. With ``n_exec`` > 1 consecutive series go to
``n_exec`` executors (clones of ``ffa``), each on its own compute stream, so
one series' brute fold (latency-bound, little HBM traffic) runs beside the
previous series' merges and scoring (HBM- and issue-bound). This is the
reference's FFAFreqSweep loop over beams or DM trials
(``lib/ffa_freq_sweep.cpp:144-195``) with its per-series host round trip
hidden behind the next search.
"""

from __future__ import annotations

import numpy as np

from . import _capi as C
from . import _device as D


class SearchPipeline:
    def __init__(self, ffa, snr_min: float, max_cands: int = 1 << 20, depth: int = 2, n_exec: int = 1):
        t = D.torch()
        self.ffa = ffa
        self.snr_min = float(snr_min)
        self.cap = int(max_cands)
        self.n_exec = max(1, int(n_exec))
        self.execs = [ffa] + [ffa.clone() for _ in range(self.n_exec - 1)]
        # an input slot per series in flight: one per executor, plus the next copy
        self.depth = max(2, int(depth), self.n_exec + 1)
        dev = f"cuda:{ffa.device_id}"
        n = ffa._cfg.nsamps
        self.compute = [t.cuda.Stream(device=dev) for _ in range(self.n_exec)]
        self.copy = t.cuda.Stream(device=dev)
        self.e = [t.empty(n, dtype=t.float32, device=dev) for _ in range(self.depth)]
        self.v = [t.empty(n, dtype=t.float32, device=dev) for _ in range(self.depth)]
        self.idx = [t.empty(self.cap, dtype=t.int32, device=dev) for _ in range(self.depth)]
        self.snr = [t.empty(self.cap, dtype=t.float32, device=dev) for _ in range(self.depth)]
        self.cnt = [t.zeros(1, dtype=t.int64, device=dev) for _ in range(self.depth)]
        self.hcnt = [t.zeros(1, dtype=t.int64).pin_memory() for _ in range(self.depth)]
        self.hidx = [t.empty(self.cap, dtype=t.int32).pin_memory() for _ in range(self.depth)]
        self.hsnr = [t.empty(self.cap, dtype=t.float32).pin_memory() for _ in range(self.depth)]
        self.copied = [t.cuda.Event() for _ in range(self.depth)]
        self.done = [t.cuda.Event() for _ in range(self.depth)]
        self.read = [t.cuda.Event() for _ in range(self.depth)]
        self.h2d_bytes = 0
        self.d2h_bytes = 0

    def _pinned(self, x):
        t = D.torch()
        if isinstance(x, t.Tensor):
            return x if x.is_pinned() else x.pin_memory()
        return t.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).pin_memory()

    def _launch(self, k: int, e_host, v_host) -> None:
        t = D.torch()
        s = k % self.depth
        c = k % self.n_exec
        compute = self.compute[c]
        with t.cuda.stream(self.copy):
            # the slot's previous search must have consumed its inputs
            self.copy.wait_event(self.done[s])
            self.e[s].copy_(e_host, non_blocking=True)
            self.v[s].copy_(v_host, non_blocking=True)
            self.copied[s].record(self.copy)
        self.h2d_bytes += 8 * self.e[s].numel()
        with t.cuda.stream(compute):
            compute.wait_event(self.copied[s])
            # the slot's previous candidates must have been read back
            compute.wait_event(self.read[s])
            C.check(C.lib().lk_ffa_search(self.execs[c]._h, self.e[s].data_ptr(), self.v[s].data_ptr(),
                                          self.snr_min, self.idx[s].data_ptr(), self.snr[s].data_ptr(),
                                          self.cap, self.cnt[s].data_ptr(), compute.cuda_stream))
            self.hcnt[s].copy_(self.cnt[s], non_blocking=True)
            self.done[s].record(compute)

    def _collect(self, k: int):
        t = D.torch()
        s = k % self.depth
        self.done[s].synchronize()
        total = int(self.hcnt[s].item())
        n = min(total, self.cap)
        with t.cuda.stream(self.copy):
            self.copy.wait_event(self.done[s])
            self.hidx[s][:n].copy_(self.idx[s][:n], non_blocking=True)
            self.hsnr[s][:n].copy_(self.snr[s][:n], non_blocking=True)
            self.read[s].record(self.copy)
        self.read[s].synchronize()
        self.d2h_bytes += 8 + 8 * n
        return self.hidx[s][:n].numpy().view(np.uint32).copy(), self.hsnr[s][:n].numpy().copy(), total

    def run(self, series):
        """Yields (indices, snr, total) per (ts_e, ts_v) of `series`, in order."""
        pending = []
        for k, (e, v) in enumerate(series):
            self._launch(k, self._pinned(e), self._pinned(v))
            pending.append(k)
            if len(pending) > self.n_exec:
                yield self._collect(pending.pop(0))
        while pending:
            yield self._collect(pending.pop(0))
