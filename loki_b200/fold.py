"""Brute fold on the GPU, mirroring ``libculoki.fold.compute_brute_fold_time_cuda``
(reference: lib/fold.cpp:13-190, lib/fold_cuda.cu; bound at
src/loki_python_cuda.cpp:95-110).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from . import _device as D


class BruteFoldCUDA:
    """Brute fold into [nsegments, nfreqs, 2, nbins] (reference ``BruteFoldCUDA<float>``)."""

    def __init__(self, freq_arr, segment_len: int, nbins: int, nsamps: int, tsamp: float,
                 t_ref: float = 0.0, device_id: int = 0):
        D.require_cuda(device_id)
        f = np.ascontiguousarray(freq_arr, dtype=np.float64).ravel()
        self._nfreq = f.size
        self._nseg = nsamps // segment_len if segment_len else 0
        self._nbins = int(nbins)
        self._nsamps = int(nsamps)
        self._device = device_id
        h = ctypes.c_void_p()
        with D.torch().cuda.device(device_id):
            C.check(C.lib().lk_brute_fold_create(f.ctypes.data, f.size, int(segment_len), int(nbins), int(nsamps),
                                                 float(tsamp), float(t_ref), device_id, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                C.lib().lk_brute_fold_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def fold_size(self) -> int:
        return self._nseg * self._nfreq * 2 * self._nbins

    def execute(self, ts_e, ts_v, fold=None):
        host = not (D.is_device_tensor(ts_e) and D.is_device_tensor(ts_v))
        e = D.to_device_f32(ts_e, self._device)
        v = D.to_device_f32(ts_v, self._device)
        if e.numel() != self._nsamps or v.numel() != self._nsamps:
            raise RuntimeError("BruteFold::execute: ts_e and ts_v must have size nsamps")
        out = fold if D.is_device_tensor(fold) else D.empty_f32(self.fold_size, self._device)
        if out.numel() < self.fold_size:
            raise RuntimeError("BruteFold::execute: fold must have size fold_size")
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_brute_fold_execute(self._h, D.ptr(e), D.ptr(v), D.ptr(out),
                                                  D.stream_ptr(self._device)))
        return out[: self.fold_size].cpu().numpy() if host else out


def compute_brute_fold_time_cuda(ts_e, ts_v, freq_arr, segment_len: int, nbins: int, tsamp: float,
                                 t_ref: float = 0.0, device_id: int = 0) -> np.ndarray:
    """Flat [nsegments * nfreqs * 2 * nbins] brute fold (float32)."""
    ts_e = np.asarray(ts_e, dtype=np.float32)
    bf = BruteFoldCUDA(freq_arr, segment_len, nbins, ts_e.size, tsamp, t_ref, device_id)
    return bf.execute(ts_e, np.asarray(ts_v, dtype=np.float32))


def compute_brute_fold_fourier_cuda(ts_e, ts_v, freq_arr, segment_len: int, nbins: int, tsamp: float,
                                    t_ref: float = 0.0, device_id: int = 0):
    """Direct transform of each segment at each frequency, [nseg, nfreqs, 2,
    nbins // 2 + 1] complex64 flattened (reference
    ``compute_brute_fold_fourier_cuda``, src/loki_python_cuda.cpp:133-146)."""
    D.require_cuda(device_id)
    host = not (D.is_device_tensor(ts_e) and D.is_device_tensor(ts_v))
    f = np.ascontiguousarray(freq_arr, dtype=np.float64).ravel()
    e = D.to_device_f32(ts_e, device_id)
    v = D.to_device_f32(ts_v, device_id)
    if e.numel() != v.numel():
        raise RuntimeError("BruteFold::execute: ts_e and ts_v must have the same size")
    nseg = e.numel() // int(segment_len) if segment_len else 0
    n = nseg * f.size * 2 * (int(nbins) // 2 + 1)
    out = D.empty_f32(2 * max(n, 1), device_id)
    with D.torch().cuda.device(device_id):
        C.check(C.lib().lk_fourier_brute_fold(D.ptr(e), D.ptr(v), e.numel(), f.ctypes.data, f.size,
                                              int(segment_len), int(nbins), float(tsamp), float(t_ref),
                                              D.ptr(out), n, device_id, D.stream_ptr(device_id)))
    if host:
        return out[: 2 * n].cpu().numpy().view(np.complex64)
    return out[: 2 * n]
