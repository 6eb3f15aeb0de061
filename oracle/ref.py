"""ctypes binding of the reference's own CPU code (``oracle/_ref``). Test infrastructure only.

``libloki_ref_parity.so`` is the reference built with pinned IEEE flags and is
the parity checker; ``libloki_ref_timing_v{3,4}.so`` carry the reference's
Release flags and serve only as the timed CPU baseline.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from .lko import COORD_DTYPE, COORD_FREQ_DTYPE

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")

u64 = ctypes.c_uint64
u32 = ctypes.c_uint32
f64 = ctypes.c_double
f32 = ctypes.c_float
vp = ctypes.c_void_p


class RefCfg(ctypes.Structure):
    _fields_ = [
        ("nsamps", u64),
        ("tsamp", f64),
        ("nbins", u64),
        ("eta", f64),
        ("nparams", u32),
        ("limits", f64 * 10),
        ("bseg_brute", u64),
        ("bseg_ffa", u64),
        ("nthreads", ctypes.c_int32),
        ("ducy_max", f64),
        ("wtsp", f64),
    ]


def _host_has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("flags"):
                    flags = set(line.split())
                    return {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
    except OSError:
        pass
    return False


def lib_path(kind: str = "parity") -> str:
    if kind == "timing":
        kind = "timing_v4" if _host_has_avx512() else "timing_v3"
    return os.path.join(REF_DIR, f"libloki_ref_{kind}.so")


def available(kind: str = "parity") -> bool:
    return os.path.exists(lib_path(kind))


_libs: dict[str, ctypes.CDLL] = {}


def lib(kind: str = "parity") -> ctypes.CDLL:
    path = lib_path(kind)
    if path not in _libs:
        if not os.path.exists(path):
            raise RuntimeError(f"reference library missing: {path} (run `make -C oracle ref`)")
        L = ctypes.CDLL(path)
        L.lkref_last_error.restype = ctypes.c_char_p
        L.lkref_max_threads.restype = ctypes.c_int
        L.lkref_ffa_create.argtypes = [vp, vp]
        L.lkref_ffa_destroy.argtypes = [vp]
        L.lkref_ffa_info.argtypes = [vp] + [vp] * 6 + [u64] + [vp] * 6
        L.lkref_ffa_execute.argtypes = [vp, vp, vp, u64, vp, u64]
        L.lkref_resolve_freq.argtypes = [vp, vp, u64]
        L.lkref_resolve.argtypes = [vp, vp, u64]
        L.lkref_brute_fold.argtypes = [vp, vp, u64, vp, u64, u64, u64, f64, f64, ctypes.c_int, vp, u64]
        L.lkref_snr_boxcar_3d.argtypes = [vp, u64, u64, vp, u64, ctypes.c_int, vp]
        L.lkref_snr_boxcar_3d_max.argtypes = [vp, u64, u64, vp, u64, ctypes.c_int, vp]
        L.lkref_box_widths.argtypes = [u64, f64, f64, vp, u64, vp]
        L.lkref_phase_idx.restype = f32
        L.lkref_phase_idx.argtypes = [f64, f64, u64, f64]
        L.lkref_phase_idx_uint.restype = u32
        L.lkref_phase_idx_uint.argtypes = [f64, f64, u64, f64]
        _libs[path] = L
    return _libs[path]


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def make_cfg(nsamps, tsamp, nbins, eta, param_limits, bseg_brute=None, bseg_ffa=None,
             nthreads=1, ducy_max=0.2, wtsp=1.5) -> RefCfg:
    lim = np.asarray(param_limits, dtype=np.float64).reshape(-1, 2)
    c = RefCfg()
    c.nsamps, c.tsamp, c.nbins, c.eta = nsamps, tsamp, nbins, eta
    c.nparams = lim.shape[0]
    for i, (a, b) in enumerate(lim):
        c.limits[2 * i] = a
        c.limits[2 * i + 1] = b
    c.bseg_brute = bseg_brute or 0
    c.bseg_ffa = bseg_ffa or 0
    c.nthreads = nthreads
    c.ducy_max, c.wtsp = ducy_max, wtsp
    return c


class RefFFA:
    """algorithms::FFA<float> of the reference, built once and executed many times."""

    def __init__(self, cfg: RefCfg, kind: str = "parity"):
        self._lib = lib(kind)
        self.cfg = cfg
        self._h = vp()
        if self._lib.lkref_ffa_create(ctypes.byref(cfg), ctypes.byref(self._h)) != 0:
            raise RuntimeError(self._lib.lkref_last_error().decode())
        L, buf, fs, bfs, cs, bb = (u64() for _ in range(6))
        m = 64
        self.segment_lens = np.zeros(m, np.uint64)
        self.nsegments = np.zeros(m, np.uint64)
        self.ncoords = np.zeros(m, np.uint64)
        self.ncoords_offsets = np.zeros(m + 1, np.uint32)
        counts = np.zeros(m * cfg.nparams, np.uint64)
        dparams = np.zeros(m * cfg.nparams, np.float64)
        rc = self._lib.lkref_ffa_info(
            self._h, *(ctypes.byref(x) for x in (L, buf, fs, bfs, cs, bb)), m,
            _p(self.segment_lens), _p(self.nsegments), _p(self.ncoords), _p(self.ncoords_offsets),
            _p(counts), _p(dparams))
        if rc != 0:
            raise RuntimeError(self._lib.lkref_last_error().decode())
        self.n_levels = L.value
        n = self.n_levels
        self.segment_lens = self.segment_lens[:n]
        self.nsegments = self.nsegments[:n]
        self.ncoords = self.ncoords[:n]
        self.ncoords_offsets = self.ncoords_offsets[: n + 1]
        self.param_counts = counts[: n * cfg.nparams].reshape(n, cfg.nparams)
        self.dparams = dparams[: n * cfg.nparams].reshape(n, cfg.nparams)
        self.buffer_size = buf.value
        self.fold_size = fs.value
        self.brute_fold_size = bfs.value
        self.coord_size = cs.value
        self.bseg_brute = bb.value
        self._fold = np.zeros(self.buffer_size, dtype=np.float32)

    def execute(self, ts_e: np.ndarray, ts_v: np.ndarray) -> np.ndarray:
        """Final-level fold (a view of an internal buffer, valid until the next call)."""
        rc = self._lib.lkref_ffa_execute(self._h, _p(ts_e), _p(ts_v), ts_e.size, _p(self._fold), self._fold.size)
        if rc != 0:
            raise RuntimeError(self._lib.lkref_last_error().decode())
        return self._fold[: self.fold_size]

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.lkref_ffa_destroy(self._h)
            self._h = None


def resolve(cfg: RefCfg, coord_size: int) -> np.ndarray:
    L = lib()
    if cfg.nparams == 1:
        out = np.zeros(coord_size, dtype=COORD_FREQ_DTYPE)
        rc = L.lkref_resolve_freq(ctypes.byref(cfg), _p(out), coord_size)
    else:
        out = np.zeros(coord_size, dtype=COORD_DTYPE)
        rc = L.lkref_resolve(ctypes.byref(cfg), _p(out), coord_size)
    if rc != 0:
        raise RuntimeError(L.lkref_last_error().decode())
    return out


def brute_fold(ts_e, ts_v, freqs, segment_len, nbins, tsamp, t_ref=0.0, nthreads=1) -> np.ndarray:
    L = lib()
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    out = np.zeros((ts_e.size // segment_len) * freqs.size * 2 * nbins, dtype=np.float32)
    rc = L.lkref_brute_fold(_p(ts_e), _p(ts_v), ts_e.size, _p(freqs), freqs.size, segment_len, nbins,
                            tsamp, t_ref, nthreads, _p(out), out.size)
    if rc != 0:
        raise RuntimeError(L.lkref_last_error().decode())
    return out


def snr_boxcar_3d(folds, widths, nbins, nthreads=1, kind="parity") -> np.ndarray:
    L = lib(kind)
    folds = np.ascontiguousarray(folds, dtype=np.float32)
    w = np.ascontiguousarray(widths, dtype=np.uint64)
    nprof = folds.size // (2 * nbins)
    out = np.zeros((nprof, w.size), dtype=np.float32)
    if L.lkref_snr_boxcar_3d(_p(folds), nprof, nbins, _p(w), w.size, nthreads, _p(out)) != 0:
        raise RuntimeError(L.lkref_last_error().decode())
    return out


def snr_boxcar_3d_max(folds, widths, nbins, nthreads=1) -> np.ndarray:
    L = lib()
    folds = np.ascontiguousarray(folds, dtype=np.float32)
    w = np.ascontiguousarray(widths, dtype=np.uint64)
    nprof = folds.size // (2 * nbins)
    out = np.zeros(nprof, dtype=np.float32)
    if L.lkref_snr_boxcar_3d_max(_p(folds), nprof, nbins, _p(w), w.size, nthreads, _p(out)) != 0:
        raise RuntimeError(L.lkref_last_error().decode())
    return out


def box_widths(nbins, ducy_max=0.2, wtsp=1.5) -> np.ndarray:
    L = lib()
    out = np.zeros(64, dtype=np.uint64)
    n = u64()
    if L.lkref_box_widths(nbins, ducy_max, wtsp, _p(out), 64, ctypes.byref(n)) != 0:
        raise RuntimeError(L.lkref_last_error().decode())
    return out[: n.value].copy()


def phase_idx(t, f, nbins, delay=0.0) -> float:
    return lib().lkref_phase_idx(t, f, nbins, delay)


def phase_idx_uint(t, f, nbins, delay=0.0) -> int:
    return lib().lkref_phase_idx_uint(t, f, nbins, delay)
