"""Boxcar S/N on the GPU, mirroring ``libculoki.scores`` / ``libloki.scores``
(reference: lib/score.cpp:95-172, 390-529; lib/score_cuda.cu;
bindings src/loki_python.cpp:71-157, src/loki_python_cuda.cpp:21-63).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from . import _device as D


def generate_box_width_trials(nbins: int, ducy_max: float = 0.3, wtsp: float = 1.5) -> np.ndarray:
    out = np.zeros(C.LK_MAX_WIDTHS, dtype=np.uint32)
    n = ctypes.c_uint32()
    C.check(C.lib().lk_box_width_trials(int(nbins), float(ducy_max), float(wtsp), out.ctypes.data,
                                        C.LK_MAX_WIDTHS, ctypes.byref(n)))
    return out[: n.value].astype(np.uint64)


def _widths(widths) -> np.ndarray:
    w = np.ascontiguousarray(widths).astype(np.uint32).ravel()
    if w.size == 0:
        raise RuntimeError("Input arrays cannot be empty")
    return w


def _run3d(arr, widths, device_id: int, mode: int):
    D.require_cuda(device_id)
    host = not D.is_device_tensor(arr)
    if host:
        a = np.asarray(arr)
        if a.ndim != 3:
            raise RuntimeError("Input array must be 3-dimensional, widths must be 1-dimensional")
        if a.shape[0] == 0 or a.shape[1] == 0:
            raise RuntimeError("Input arrays cannot be empty")
        nprof, nbins = a.shape[0], a.shape[2]
    else:
        if arr.dim() != 3:
            raise RuntimeError("Input array must be 3-dimensional, widths must be 1-dimensional")
        nprof, nbins = arr.shape[0], arr.shape[2]
    w = _widths(widths)
    d = D.to_device_f32(arr, device_id)
    nout = nprof * (w.size if mode == C.LK_SCORE_PER_WIDTH else 1)
    out = D.empty_f32(nout, device_id)
    with D.torch().cuda.device(device_id):
        C.check(C.lib().lk_snr_boxcar_3d(D.ptr(d), nprof, nbins, w.ctypes.data, w.size, mode, D.ptr(out),
                                         D.stream_ptr(device_id)))
    shape = (nprof, w.size) if mode == C.LK_SCORE_PER_WIDTH else (nprof,)
    return out.cpu().numpy().reshape(shape) if host else out.reshape(shape)


def snr_boxcar_3d(arr, widths, device_id: int = 0):
    """S/N per width of [nprofiles, 2, nbins] (E, V) folds -> [nprofiles, nwidths]."""
    return _run3d(arr, widths, device_id, C.LK_SCORE_PER_WIDTH)


def snr_boxcar_3d_max(arr, widths, device_id: int = 0):
    """Maximum S/N over widths of [nprofiles, 2, nbins] folds -> [nprofiles]."""
    return _run3d(arr, widths, device_id, C.LK_SCORE_MAX)


def snr_boxcar_2d_max(arr, widths, stdnoise: float = 1.0, device_id: int = 0):
    """Maximum S/N over widths of [nprofiles, nbins] profiles, divided by stdnoise."""
    D.require_cuda(device_id)
    host = not D.is_device_tensor(arr)
    shape = np.asarray(arr).shape if host else tuple(arr.shape)
    if len(shape) != 2:
        raise RuntimeError("Input array must be 2-dimensional, widths must be 1-dimensional")
    if shape[0] == 0 or shape[1] == 0:
        raise RuntimeError("Input arrays cannot be empty")
    nprof, nbins = shape
    w = _widths(widths)
    d = D.to_device_f32(arr, device_id)
    out = D.empty_f32(nprof, device_id)
    with D.torch().cuda.device(device_id):
        C.check(C.lib().lk_snr_boxcar_2d_max(D.ptr(d), nprof, nbins, w.ctypes.data, w.size, float(stdnoise),
                                             D.ptr(out), D.stream_ptr(device_id)))
    return out.cpu().numpy() if host else out


def compact_ge(scores, thr: float, max_out: int | None = None, device_id: int = 0):
    """Indices and values of scores >= thr, in increasing index order, and the
    total count passing (FFAFreqSweep compaction, lib/ffa_freq_sweep.cpp:182-195)."""
    D.require_cuda(device_id)
    t = D.torch()
    s = D.to_device_f32(scores, device_id).reshape(-1)
    n = s.numel()
    cap = n if max_out is None else int(max_out)
    idx = t.empty(max(cap, 1), dtype=t.int32, device=f"cuda:{device_id}")
    val = D.empty_f32(max(cap, 1), device_id)
    cnt = t.zeros(1, dtype=t.int64, device=f"cuda:{device_id}")
    scratch = t.empty(int(C.lib().lk_compact_scratch_bytes(n)), dtype=t.uint8, device=f"cuda:{device_id}")
    with t.cuda.device(device_id):
        C.check(C.lib().lk_compact_ge(D.ptr(s), n, float(thr), idx.data_ptr(), D.ptr(val), cap, cnt.data_ptr(),
                                      scratch.data_ptr(), D.stream_ptr(device_id)))
    total = int(cnt.item())
    k = min(total, cap)
    return idx[:k].cpu().numpy().view(np.uint32), val[:k].cpu().numpy(), total
