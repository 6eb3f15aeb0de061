"""FFA on the GPU: ``FFACUDA`` (time domain), ``FFACOMPLEXCUDA`` (Fourier
domain), ``compute_ffa_time_cuda``, ``compute_ffa_fourier_cuda``,
``compute_ffa_fourier_return_to_time_cuda`` and ``compute_ffa_scores_cuda``,
mirroring ``libculoki.ffa`` of the reference (src/loki_python_cuda.cpp:148-204,
lib/ffa_cuda.cu:609-692).

Inputs may be host arrays (copied in, results copied back, as the
reference's host-span overloads do) or CUDA tensors (work is enqueued on the
current torch stream and device tensors are returned, as the reference's
device-span overloads do).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from . import _device as D
from .configs import PulsarSearchConfig
from .plans import FFAPlanFourier, FFAPlanTime

_STORAGE = {"fp32": C.LK_FP32, "float32": C.LK_FP32, "bf16": C.LK_BF16, "fp16": C.LK_FP16}


class FFACUDA:
    """Time-domain FFA executor on one device (reference ``FFACUDA<float>``).

    The executor owns the coordinate tables, brute-fold run tables and the
    intermediate fold buffers; it can be executed many times.
    """

    def __init__(self, cfg: PulsarSearchConfig, device_id: int = 0, fold_storage: str = "fp32",
                 max_batch: int = 1):
        D.require_cuda(device_id)
        self._cfg = cfg
        self._plan = FFAPlanTime(cfg)
        self._device = device_id
        self._max_batch = int(max_batch)
        self._storage = fold_storage
        if fold_storage not in _STORAGE:
            raise ValueError(f"fold_storage must be one of {sorted(_STORAGE)}")
        h = ctypes.c_void_p()
        with D.torch().cuda.device(device_id):
            C.check(C.lib().lk_ffa_create_batched(cfg._plan_handle, device_id, _STORAGE[fold_storage],
                                                  self._max_batch, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                C.lib().lk_ffa_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def plan(self) -> FFAPlanTime:
        return self._plan

    @property
    def fold_storage(self) -> str:
        return self._storage

    def clone(self) -> "FFACUDA":
        """A second executor of the same configuration, storage and tuning
        (its own buffers, so the two can search on different streams)."""
        other = FFACUDA(self._cfg, self._device, self._storage, self._max_batch)
        other.set_tuning(self.tuning)
        if self._storage == "bf16":
            other.set_rescore_margin(*self.rescore_margin)
        return other

    @property
    def device_id(self) -> int:
        return self._device

    @property
    def workspace_bytes(self) -> int:
        n = ctypes.c_uint64()
        C.check(C.lib().lk_ffa_workspace_bytes(self._h, ctypes.byref(n)))
        return n.value

    def _inputs(self, ts_e, ts_v):
        n = self._cfg.nsamps
        e = D.to_device_f32(ts_e, self._device)
        v = D.to_device_f32(ts_v, self._device)
        if e.numel() != n:
            raise RuntimeError("FFA::execute: ts_e must have size nsamps")
        if v.numel() != e.numel():
            raise RuntimeError("FFA::execute: ts_v must have size nsamps")
        return e, v

    def execute(self, ts_e, ts_v, fold=None):
        """Final-level fold. With a CUDA tensor `fold` (>= fold_size floats) the
        result is written there; otherwise a new array/tensor is returned."""
        host = not (D.is_device_tensor(ts_e) and D.is_device_tensor(ts_v))
        e, v = self._inputs(ts_e, ts_v)
        n = self._plan.fold_size
        out = fold if D.is_device_tensor(fold) else D.empty_f32(n, self._device)
        if out.numel() < n:
            raise RuntimeError("FFA::execute: fold must have size >= fold_size")
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_ffa_execute(self._h, D.ptr(e), D.ptr(v), D.ptr(out), out.numel(),
                                           D.stream_ptr(self._device)))
        if fold is not None and not D.is_device_tensor(fold):
            np.copyto(np.asarray(fold).reshape(-1)[:n], out[:n].cpu().numpy())
            return fold
        return out[:n].cpu().numpy() if host else out

    @property
    def scores_exact(self) -> bool:
        """Whether scores() equals the FP32 (reference) S/N bit for bit: True
        for FP32 storage. With BF16 storage the S/N values carry the storage
        error (RMS ~0.008, at most ~0.06 on the 2^22-sample accelerated
        search against FP64); search() still returns the FP32 candidates and
        S/N, rescoring every cell near the threshold exactly."""
        return self._storage == "fp32"

    def scores(self, ts_e, ts_v, out=None):
        """Boxcar S/N [ncoords_final, n_widths] (final level fused with scoring).
        With fold_storage="bf16" these are approximations (see scores_exact);
        candidates come exact from search()."""
        host = not (D.is_device_tensor(ts_e) and D.is_device_tensor(ts_v))
        e, v = self._inputs(ts_e, ts_v)
        nc = int(self._plan.ncoords[-1])
        nw = self._cfg.n_scoring_widths
        res = out if D.is_device_tensor(out) else D.empty_f32(nc * nw, self._device)
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_ffa_scores(self._h, D.ptr(e), D.ptr(v), D.ptr(res), res.numel(),
                                          D.stream_ptr(self._device)))
        if host:
            return res[: nc * nw].cpu().numpy()
        return res

    def search(self, ts_e, ts_v, snr_min: float | None = None, max_cands: int | None = None):
        """Scores compacted to ``score >= snr_min`` in flat (coord * n_widths + width)
        order, as FFAFreqSweep does. Returns (indices, snrs, n_total_passing)."""
        e, v = self._inputs(ts_e, ts_v)
        thr = self._cfg.snr_min if snr_min is None else float(snr_min)
        cap = self._cfg.max_passing_candidates if max_cands is None else int(max_cands)
        t = D.torch()
        idx = t.empty(cap, dtype=t.int32, device=f"cuda:{self._device}")
        snr = D.empty_f32(cap, self._device)
        cnt = t.zeros(1, dtype=t.int64, device=f"cuda:{self._device}")
        with t.cuda.device(self._device):
            C.check(C.lib().lk_ffa_search(self._h, D.ptr(e), D.ptr(v), thr, idx.data_ptr(), D.ptr(snr),
                                          cap, cnt.data_ptr(), D.stream_ptr(self._device)))
        total = int(cnt.item())
        k = min(total, cap)
        return idx[:k].cpu().numpy().view(np.uint32), snr[:k].cpu().numpy(), total

    # ---- batches of equal-length series ([nbatch, nsamps] CUDA tensors) -------------

    def _batch_inputs(self, ts_e, ts_v):
        n = self._cfg.nsamps
        e = D.to_device_f32(ts_e, self._device).reshape(-1)
        v = D.to_device_f32(ts_v, self._device).reshape(-1)
        if e.numel() % n != 0 or e.numel() != v.numel():
            raise RuntimeError("batch inputs must be [nbatch, nsamps] with matching ts_e / ts_v")
        nb = e.numel() // n
        if nb < 1 or nb > self._max_batch:
            raise RuntimeError(f"nbatch must lie in [1, max_batch={self._max_batch}]")
        return e, v, nb

    def execute_batch(self, ts_e, ts_v, out=None):
        """Final-level fold of each series of the batch: a [nbatch, fold_size]
        CUDA tensor (one launch per level for the whole batch)."""
        e, v, nb = self._batch_inputs(ts_e, ts_v)
        per = int(self._plan.fold_size)
        res = out if out is not None else D.empty_f32(nb * per, self._device)
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_ffa_execute_batch(self._h, D.ptr(e), D.ptr(v), nb, D.ptr(res), res.numel(),
                                                 D.stream_ptr(self._device)))
        return res.reshape(nb, per) if out is None else res

    def scores_batch(self, ts_e, ts_v, out=None):
        """Boxcar S/N of each series of the batch: a [nbatch, ncoords_final *
        n_widths] CUDA tensor (one launch per level for the whole batch)."""
        e, v, nb = self._batch_inputs(ts_e, ts_v)
        per = int(self._plan.ncoords[-1]) * self._cfg.n_scoring_widths
        res = out if out is not None else D.empty_f32(nb * per, self._device)
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_ffa_scores_batch(self._h, D.ptr(e), D.ptr(v), nb, D.ptr(res), res.numel(),
                                                D.stream_ptr(self._device)))
        return res.reshape(nb, per) if out is None else res

    def search_batch(self, ts_e, ts_v, snr_min: float | None = None, idx=None, snr=None, count=None):
        """Scores of the batch compacted to S/N >= snr_min in flat
        ((series * ncoords + coord) * n_widths + width) order. With idx / snr /
        count CUDA tensors given, nothing is allocated (graph-capturable) and
        they are returned; otherwise returns host (indices, snrs, total)."""
        e, v, nb = self._batch_inputs(ts_e, ts_v)
        thr = self._cfg.snr_min if snr_min is None else float(snr_min)
        t = D.torch()
        given = idx is not None
        if not given:
            cap = self._cfg.max_passing_candidates
            idx = t.empty(cap, dtype=t.int32, device=f"cuda:{self._device}")
            snr = D.empty_f32(cap, self._device)
            count = t.zeros(1, dtype=t.int64, device=f"cuda:{self._device}")
        with t.cuda.device(self._device):
            C.check(C.lib().lk_ffa_search_batch(self._h, D.ptr(e), D.ptr(v), nb, thr, idx.data_ptr(),
                                                D.ptr(snr), idx.numel(), count.data_ptr(),
                                                D.stream_ptr(self._device)))
        if given:
            return idx, snr, count
        total = int(count.item())
        k = min(total, idx.numel())
        return idx[:k].cpu().numpy().view(np.uint32), snr[:k].cpu().numpy(), total

    def set_batch_lengths(self, lengths) -> None:
        """Valid samples of each series of the next batched calls: a CUDA
        int64 tensor (one entry per series, read by every launch, so a
        captured graph sees values written into it later) or None (off).
        Samples at or past a series' length must be zero; the brute fold
        then skips the segments holding none of its samples and sets their
        folds to +0.0 (the folds of zeros), so outputs do not change."""
        if lengths is None:
            self._batch_lengths = None
            C.check(C.lib().lk_ffa_set_batch_lengths(self._h, None))
            return
        if not D.is_device_tensor(lengths) or lengths.dtype != D.torch().int64 or not lengths.is_contiguous():
            raise ValueError("lengths must be a contiguous int64 CUDA tensor")
        self._batch_lengths = lengths  # kept alive while the executor reads it
        C.check(C.lib().lk_ffa_set_batch_lengths(self._h, D.ptr(lengths)))

    def set_profiling(self, enable: bool = True) -> None:
        """Record CUDA events around every kernel stage of subsequent calls."""
        C.check(C.lib().lk_ffa_set_profiling(self._h, 1 if enable else 0))

    def profile(self) -> list[dict]:
        """Stages of the last call: kind, level, launches, GPU ms, algorithmic bytes."""
        arr = (C.LkStageTime * 128)()
        n = ctypes.c_uint32()
        C.check(C.lib().lk_ffa_get_profile(self._h, D.stream_ptr(self._device), arr, 128, ctypes.byref(n)))
        return [
            {"stage": C.STAGE_NAMES.get(arr[i].kind, str(arr[i].kind)), "level": arr[i].level,
             "launches": arr[i].launches, "ms": float(arr[i].ms), "bytes": int(arr[i].bytes)}
            for i in range(min(n.value, 128))
        ]

    def status(self) -> int:
        st = ctypes.c_uint32()
        C.check(C.lib().lk_ffa_status(self._h, D.stream_ptr(self._device), ctypes.byref(st)))
        return st.value

    _TUNING_FIELDS = ("bf_rows", "bf_warps", "bf_stages", "merge_rows_in_flight", "score_cells_per_block",
                      "bf_tmem_warps")

    def autotune(self, ts_e, ts_v, reps: int = 3) -> dict:
        """Time launch-shape candidates of the brute fold, the merges and the
        fused final level (plans with one final segment) on this series (CUDA
        tensors or host arrays) and keep the fastest of each; results are
        unchanged. Returns the tuning with the best stage times (ms)."""
        e, v = self._inputs(ts_e, ts_v)
        t = C.LkTuning()
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_ffa_autotune(self._h, D.ptr(e), D.ptr(v), int(reps), ctypes.byref(t),
                                            D.stream_ptr(self._device)))
        return {name: getattr(t, name) for name, _ in C.LkTuning._fields_}

    @property
    def tuning(self) -> dict:
        t = C.LkTuning()
        C.check(C.lib().lk_ffa_get_tuning(self._h, ctypes.byref(t)))
        return {name: getattr(t, name) for name, _ in C.LkTuning._fields_}

    def set_tuning(self, tuning: dict) -> None:
        """Apply a tuning returned by ``autotune`` / ``tuning`` (launch shapes only)."""
        t = C.LkTuning()
        for name in self._TUNING_FIELDS:
            setattr(t, name, int(tuning.get(name, 0)))
        C.check(C.lib().lk_ffa_set_tuning(self._h, ctypes.byref(t)))

    @property
    def rescore_margin(self) -> tuple[float, float]:
        """BF16 search margin (abs, rel): cells with approximate best S/N >=
        (snr_min - abs) / (1 + rel) are rescored exactly."""
        a, r = ctypes.c_float(), ctypes.c_float()
        C.check(C.lib().lk_ffa_get_rescore_margin(self._h, ctypes.byref(a), ctypes.byref(r)))
        return float(a.value), float(r.value)

    def set_rescore_margin(self, margin_abs: float, margin_rel: float) -> None:
        C.check(C.lib().lk_ffa_set_rescore_margin(self._h, float(margin_abs), float(margin_rel)))

    def rescored_cells(self) -> int:
        """Final cells the last BF16 search rescored exactly."""
        n = ctypes.c_uint64()
        C.check(C.lib().lk_ffa_rescored_cells(self._h, D.stream_ptr(self._device), ctypes.byref(n)))
        return int(n.value)


def compute_ffa_time_cuda(ts_e, ts_v, cfg: PulsarSearchConfig, device_id: int = 0, quiet: bool = False):
    """Final-level time-domain fold and its plan (reference lib/ffa_cuda.cu:609-628)."""
    ffa = FFACUDA(cfg, device_id)
    return ffa.execute(np.asarray(ts_e, dtype=np.float32), np.asarray(ts_v, dtype=np.float32)), ffa.plan


def compute_ffa_fourier_cuda(ts_e, ts_v, cfg: PulsarSearchConfig, device_id: int = 0, quiet: bool = False):
    """Final-level Fourier-domain fold (complex64, flattened) and its plan
    (reference compute_ffa_cuda<ComplexTypeCUDA>, lib/ffa_cuda.cu:629-650)."""
    ffa = FFACOMPLEXCUDA(cfg, device_id)
    return ffa.execute(np.asarray(ts_e, dtype=np.float32), np.asarray(ts_v, dtype=np.float32)), ffa.plan


def compute_ffa_fourier_return_to_time_cuda(ts_e, ts_v, cfg: PulsarSearchConfig, device_id: int = 0,
                                            quiet: bool = False):
    """Final-level fold of the Fourier-domain FFA back in time and the
    time-domain plan (reference lib/ffa_cuda.cu:651-670)."""
    ffa = FFACOMPLEXCUDA(cfg, device_id)
    fold = ffa.execute_time(np.asarray(ts_e, dtype=np.float32), np.asarray(ts_v, dtype=np.float32))
    return fold, FFAPlanTime(cfg)


def compute_ffa_scores_cuda(ts_e, ts_v, cfg: PulsarSearchConfig, device_id: int = 0, quiet: bool = False):
    """Boxcar S/N of every final coordinate and width, and the time-domain
    plan (reference lib/ffa_cuda.cu:671-692): through the Fourier-domain FFA
    when ``cfg.use_fourier`` (the reference default), else the time domain."""
    e = np.asarray(ts_e, dtype=np.float32)
    v = np.asarray(ts_v, dtype=np.float32)
    if cfg.use_fourier:
        ffa = FFACOMPLEXCUDA(cfg, device_id)
        return ffa.scores(e, v), FFAPlanTime(cfg)
    ffa = FFACUDA(cfg, device_id)
    return ffa.scores(e, v), ffa.plan


class FFACOMPLEXCUDA:
    """Fourier-domain FFA executor on one device (reference
    ``FFACUDA<ComplexTypeCUDA>``, bound as ``FFACOMPLEXCUDA``): folds are
    nbins // 2 + 1 complex harmonics, merges rotate them by the fractional
    shifts, results return to time by an inverse real transform. Level 0 is
    the direct transform of each segment for nbins <= cfg.nbins_min_lossy_bf,
    else the time-domain brute fold and a real transform."""

    def __init__(self, cfg: PulsarSearchConfig, device_id: int = 0):
        D.require_cuda(device_id)
        self._cfg = cfg
        self._plan = FFAPlanFourier(cfg)
        self._device = device_id
        h = ctypes.c_void_p()
        with D.torch().cuda.device(device_id):
            C.check(C.lib().lk_fourier_create(cfg._plan_handle, device_id, int(cfg.nbins_min_lossy_bf),
                                              ctypes.byref(h)))
        self._h = h
        nbf, fs, fst, ws = (ctypes.c_uint64() for _ in range(4))
        lossy = ctypes.c_int()
        C.check(C.lib().lk_fourier_info(h, ctypes.byref(nbf), ctypes.byref(fs), ctypes.byref(fst),
                                        ctypes.byref(lossy), ctypes.byref(ws)))
        self._fold_size, self._fold_size_time = int(fs.value), int(fst.value)
        self.lossy = bool(lossy.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                C.lib().lk_fourier_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def plan(self) -> FFAPlanFourier:
        return self._plan

    @property
    def device_id(self) -> int:
        return self._device

    @property
    def workspace_bytes(self) -> int:
        n = ctypes.c_uint64()
        C.check(C.lib().lk_fourier_info(self._h, None, None, None, None, ctypes.byref(n)))
        return int(n.value)

    def _inputs(self, ts_e, ts_v):
        n = self._cfg.nsamps
        e = D.to_device_f32(ts_e, self._device)
        v = D.to_device_f32(ts_v, self._device)
        if e.numel() != n:
            raise RuntimeError("FFA::execute: ts_e must have size nsamps")
        if v.numel() != e.numel():
            raise RuntimeError("FFA::execute: ts_v must have size nsamps")
        return e, v

    def execute(self, ts_e, ts_v, fold=None):
        """Final complex fold [nseg, ncoords, 2, nbins_f], flattened. A host
        ``fold`` of complex64 receives the complex fold; one of float32
        receives the fold back in time (the reference's two overloads). A CUDA
        tensor ``fold`` (float32, 2 * fold_size values) receives the complex
        fold as interleaved (re, im). Without ``fold`` a complex64 array (host
        inputs) or an interleaved float32 tensor (CUDA inputs) is returned."""
        if fold is not None and not D.is_device_tensor(fold) and np.asarray(fold).dtype == np.float32:
            out = self.execute_time(ts_e, ts_v)
            np.copyto(np.asarray(fold).reshape(-1)[: out.size], out)
            return fold
        host = not (D.is_device_tensor(ts_e) and D.is_device_tensor(ts_v))
        e, v = self._inputs(ts_e, ts_v)
        n = self._fold_size
        out = fold if D.is_device_tensor(fold) else D.empty_f32(2 * n, self._device)
        if out.numel() < 2 * n:
            raise RuntimeError("FFA::execute: fold must have size >= 2 * fold_size")
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_fourier_execute(self._h, D.ptr(e), D.ptr(v), D.ptr(out), out.numel() // 2,
                                               D.stream_ptr(self._device)))
        if fold is not None and not D.is_device_tensor(fold):
            np.copyto(np.asarray(fold).reshape(-1)[:n], out[: 2 * n].cpu().numpy().view(np.complex64))
            return fold
        return out[: 2 * n].cpu().numpy().view(np.complex64) if host else out[: 2 * n]

    def execute_time(self, ts_e, ts_v, fold=None):
        """Final fold back in time [nseg, ncoords, 2, nbins] float32, flattened."""
        host = not (D.is_device_tensor(ts_e) and D.is_device_tensor(ts_v))
        e, v = self._inputs(ts_e, ts_v)
        n = self._fold_size_time
        out = fold if D.is_device_tensor(fold) else D.empty_f32(n, self._device)
        if out.numel() < n:
            raise RuntimeError("FFA::execute: fold must have size >= fold_size_time")
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_fourier_execute_time(self._h, D.ptr(e), D.ptr(v), D.ptr(out), out.numel(),
                                                    D.stream_ptr(self._device)))
        return out[:n].cpu().numpy() if host else out[:n]

    def scores(self, ts_e, ts_v, out=None):
        """Boxcar S/N [ncoords_final * n_widths] of the fold back in time."""
        host = not (D.is_device_tensor(ts_e) and D.is_device_tensor(ts_v))
        e, v = self._inputs(ts_e, ts_v)
        nc = int(self._plan.ncoords[-1])
        nw = self._cfg.n_scoring_widths
        res = out if D.is_device_tensor(out) else D.empty_f32(nc * nw, self._device)
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_fourier_scores(self._h, D.ptr(e), D.ptr(v), D.ptr(res), res.numel(),
                                              D.stream_ptr(self._device)))
        return res[: nc * nw].cpu().numpy() if host else res

    def search(self, ts_e, ts_v, snr_min: float | None = None, max_cands: int | None = None):
        """Scores compacted to ``score >= snr_min`` in flat order. Returns
        (indices, snrs, n_total_passing)."""
        e, v = self._inputs(ts_e, ts_v)
        thr = self._cfg.snr_min if snr_min is None else float(snr_min)
        cap = self._cfg.max_passing_candidates if max_cands is None else int(max_cands)
        t = D.torch()
        idx = t.empty(cap, dtype=t.int32, device=f"cuda:{self._device}")
        snr = D.empty_f32(cap, self._device)
        cnt = t.zeros(1, dtype=t.int64, device=f"cuda:{self._device}")
        with t.cuda.device(self._device):
            C.check(C.lib().lk_fourier_search(self._h, D.ptr(e), D.ptr(v), thr, idx.data_ptr(), D.ptr(snr), cap,
                                              cnt.data_ptr(), D.stream_ptr(self._device)))
        total = int(cnt.item())
        k = min(total, cap)
        return idx[:k].cpu().numpy().view(np.uint32), snr[:k].cpu().numpy(), total

    _LEVEL0 = {"auto": 0, "cuda_cores": 1, "tensor_cores": 2}

    def set_level0(self, mode: str = "auto") -> None:
        """Kernel of the level-0 direct transform: "auto" (the tensor cores when
        the shape allows), "cuda_cores" or "tensor_cores"."""
        C.check(C.lib().lk_fourier_set_level0(self._h, self._LEVEL0[mode]))

    def autotune(self, ts_e, ts_v, reps: int = 3) -> float:
        """Time the tensor-core level 0's tilings on this series and keep the
        fastest; returns its time (ms), 0 when level 0 is not on the tensor
        cores. Results agree to FP32 accuracy whichever is kept."""
        e, v = self._inputs(ts_e, ts_v)
        ms = ctypes.c_float()
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_fourier_autotune(self._h, D.ptr(e), D.ptr(v), int(reps), ctypes.byref(ms),
                                                D.stream_ptr(self._device)))
        return float(ms.value)

    @property
    def level0(self) -> str:
        """Level-0 kernel in use: "tensor_cores", "cuda_cores" or "lossy"."""
        m = ctypes.c_int()
        C.check(C.lib().lk_fourier_get_level0(self._h, ctypes.byref(m)))
        return {0: "lossy", 1: "cuda_cores", 2: "tensor_cores"}[m.value]

    def status(self) -> int:
        """Device status word (bits set by bounded waits that gave up)."""
        st = ctypes.c_uint32()
        C.check(C.lib().lk_fourier_status(self._h, D.stream_ptr(self._device), ctypes.byref(st)))
        return st.value

    def set_profiling(self, enable: bool = True) -> None:
        C.check(C.lib().lk_fourier_set_profiling(self._h, 1 if enable else 0))

    def profile(self) -> list[dict]:
        arr = (C.LkStageTime * 128)()
        n = ctypes.c_uint32()
        C.check(C.lib().lk_fourier_get_profile(self._h, D.stream_ptr(self._device), arr, 128, ctypes.byref(n)))
        return [
            {"stage": C.STAGE_NAMES.get(arr[i].kind, str(arr[i].kind)), "level": arr[i].level,
             "launches": arr[i].launches, "ms": float(arr[i].ms), "bytes": int(arr[i].bytes)}
            for i in range(min(n.value, 128))
        ]


from .sweep import FFAFreqSweepCUDA  # noqa: E402  (the reference binds it in the ffa submodule)
