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


_GPU_LIB = os.path.join(REF_DIR, "libloki_ref_cuda.so")
_gpu_lib = None


def gpu_available() -> bool:
    """The reference's GPU FFA library (make -C oracle refgpu) is built."""
    return os.path.exists(_GPU_LIB)


def gpu_lib() -> ctypes.CDLL:
    global _gpu_lib
    if _gpu_lib is None:
        if not gpu_available():
            raise RuntimeError(f"reference GPU library missing: {_GPU_LIB} (run `make -C oracle refgpu`)")
        L = ctypes.CDLL(_GPU_LIB)
        L.lkrefg_last_error.restype = ctypes.c_char_p
        L.lkrefg_create.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
        L.lkrefg_destroy.argtypes = [vp]
        L.lkrefg_info.argtypes = [vp, vp, vp, vp]
        L.lkrefg_scores.argtypes = [vp, vp, vp, u64, vp, vp, u64, vp, vp]
        _gpu_lib = L
    return _gpu_lib


class RefGPU:
    """The reference's own GPU path: FFACUDA<float> (or <ComplexTypeCUDA>)
    ::execute on device spans, then snr_boxcar_3d_cuda_d, enqueued on a
    stream. Device pointers are plain integers (e.g. torch data_ptr())."""

    def __init__(self, cfg: "RefCfg", device: int = 0, use_fourier: bool = False):
        self._lib = gpu_lib()
        self._h = vp()
        if self._lib.lkrefg_create(ctypes.byref(cfg), device, int(bool(use_fourier)), ctypes.byref(self._h)) != 0:
            raise RuntimeError(self._lib.lkrefg_last_error().decode())
        fl, fst, nc = u64(), u64(), u64()
        self._lib.lkrefg_info(self._h, ctypes.byref(fl), ctypes.byref(fst), ctypes.byref(nc))
        self.fold_len, self.fold_size_time, self.ncoords_final = fl.value, fst.value, nc.value

    def scores(self, d_e: int, d_v: int, nsamps: int, d_fold: int, d_widths: int, nw: int, d_scores: int,
               stream: int) -> None:
        if self._lib.lkrefg_scores(self._h, d_e, d_v, nsamps, d_fold, d_widths, nw, d_scores, stream) != 0:
            raise RuntimeError(self._lib.lkrefg_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.lkrefg_destroy(self._h)
            self._h = None


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
        L.lkref_brute_fold_complex.argtypes = [vp, vp, u64, vp, u64, u64, u64, f64, f64, ctypes.c_int, vp, u64]
        L.lkref_fourier_create.argtypes = [vp, vp]
        L.lkref_fourier_destroy.argtypes = [vp]
        L.lkref_fourier_info.argtypes = [vp, vp, vp, vp]
        L.lkref_fourier_execute.argtypes = [vp, vp, vp, u64, vp, u64]
        L.lkref_fourier_execute_time.argtypes = [vp, vp, vp, u64, vp, u64]
        L.lkref_fourier_scores.argtypes = [vp, vp, vp, u64, vp, u64]
        L.lkref_snr_boxcar_3d.argtypes = [vp, u64, u64, vp, u64, ctypes.c_int, vp]
        L.lkref_snr_boxcar_3d_max.argtypes = [vp, u64, u64, vp, u64, ctypes.c_int, vp]
        L.lkref_box_widths.argtypes = [u64, f64, f64, vp, u64, vp]
        L.lkref_phase_idx.restype = f32
        L.lkref_phase_idx.argtypes = [f64, f64, u64, f64]
        L.lkref_phase_idx_uint.restype = u32
        L.lkref_phase_idx_uint.argtypes = [f64, f64, u64, f64]
        L.lkref_middle_out.argtypes = [u64, u64, f64, u64, vp]
        L.lkref_taylor_seed.argtypes = [vp, vp, u64, vp]
        L.lkref_taylor_branch.argtypes = [vp, u64, u32, f64, f64, u64, f64, u64, vp, vp, vp]
        L.lkref_taylor_resolve.argtypes = [vp, vp, u64, vp, vp, vp]
        L.lkref_taylor_transform.argtypes = [vp, u64, vp, u64, u32, f64, f64, f64, f64, ctypes.c_int]
        L.lkref_shift_add_batch.argtypes = [vp, vp, vp, vp, vp, vp, u64, u64, u64, u64]
        L.lkref_score_filter.argtypes = [vp, u64, u64, vp, u64, f32, vp, vp, vp]
        L.lkref_branch_max.argtypes = [vp, ctypes.c_int, vp]
        L.lkref_snr_threshold.argtypes = [vp, u64, u64, vp, u64, vp, f32, vp]
        L.lkref_branching_pattern.argtypes = [vp, ctypes.c_int, u64, vp, u64, vp]
        L.lkref_branching_pattern_basis.argtypes = [vp, ctypes.c_int, ctypes.c_int, u64, vp, u64, vp]
        L.lkref_taylor_to_cheby.argtypes = [vp, u64, u32, f64, f64]
        L.lkref_cheby_to_taylor.argtypes = [vp, u64, u32, f64, f64]
        L.lkref_cheby_branch.argtypes = [vp, u64, u32, f64, f64, f64, f64, u64, f64, u64, vp, vp, vp]
        L.lkref_cheby_resolve.argtypes = [vp, vp, u64, vp, vp, vp]
        L.lkref_cheby_transform.argtypes = [vp, u64, vp, u64, u32, f64, f64, f64, f64]
        L.lkref_prune_run.argtypes = [vp, ctypes.c_int, vp, u64, vp, u64, u64, u64, u64, u64, u64,
                                      vp, vp, vp, vp, vp, u64, vp]
        L.lkref_prune_run_basis.argtypes = [ctypes.c_int, vp, ctypes.c_int, vp, u64, vp, u64, u64, u64, u64, u64, u64,
                                      vp, vp, vp, vp, vp, u64, vp]
        L.lkref_prune_run_full.argtypes = [ctypes.c_int, vp, ctypes.c_int, vp, u64, vp, u64, u64, u64, u64, u64,
                                           u64, vp, vp, vp, vp, vp, vp, u64, vp]
        L.lkref_region_plan.argtypes = [vp, f64, f64, u64, u64, ctypes.c_int, vp, u64, vp, vp]
        L.lkref_region_plan_typed.argtypes = [vp, f64, f64, u64, u64, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp,
                                              u64, vp, vp]
        L.lkref_dts_thresholds.argtypes = [f32, f32, u64, vp]
        L.lkref_dts_probs.argtypes = [u64, f32, vp]
        L.lkref_dts_profile.argtypes = [u64, f32, f32, vp]
        L.lkref_dts_bound.argtypes = [u64, f32, vp]
        L.lkref_dts_neighbours.argtypes = [vp, u64, u64, u64, vp, vp]
        L.lkref_dts_lower_bin.restype = ctypes.c_int64
        L.lkref_dts_lower_bin.argtypes = [vp, u64, f32]
        L.lkref_dts_gen_next.argtypes = [vp, f32, f32, f32, f32, vp]
        L.lkref_dts_best_path.argtypes = [vp, u64, vp, u64, vp, u64, f32, vp, vp]
        L.lkref_dts_run.argtypes = [vp, u64, f32, u64, u64, u64, f32, f32, u64, f32, f32, f32, u64, u64, vp, vp,
                                    u64, vp]
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


class RefFourier:
    """algorithms::FFA<ComplexType> of the reference (the Fourier-domain FFA)."""

    def __init__(self, cfg: RefCfg, kind: str = "parity"):
        self._lib = lib(kind)
        self.cfg = cfg
        self._h = vp()
        _check(self._lib, self._lib.lkref_fourier_create(ctypes.byref(cfg), ctypes.byref(self._h)))
        buf, fs, fst = u64(), u64(), u64()
        _check(self._lib, self._lib.lkref_fourier_info(self._h, ctypes.byref(buf), ctypes.byref(fs),
                                                       ctypes.byref(fst)))
        self.buffer_size, self.fold_size, self.fold_size_time = buf.value, fs.value, fst.value
        self._fold = np.zeros(self.buffer_size, dtype=np.complex64)
        self._tfold = np.zeros(2 * self.buffer_size, dtype=np.float32)

    def execute(self, ts_e, ts_v) -> np.ndarray:
        """Final complex fold (a view of an internal buffer, valid until the next call)."""
        _check(self._lib, self._lib.lkref_fourier_execute(self._h, _p(ts_e), _p(ts_v), ts_e.size, _p(self._fold),
                                                          self._fold.size))
        return self._fold[: self.fold_size]

    def execute_time(self, ts_e, ts_v) -> np.ndarray:
        """Final fold back in time (a view of an internal buffer)."""
        _check(self._lib, self._lib.lkref_fourier_execute_time(self._h, _p(ts_e), _p(ts_v), ts_e.size,
                                                               _p(self._tfold), self._tfold.size))
        return self._tfold[: self.fold_size_time]

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.lkref_fourier_destroy(self._h)
            self._h = None


def fourier_scores(cfg: RefCfg, ts_e, ts_v, n_scores: int, kind: str = "parity") -> np.ndarray:
    """compute_ffa_scores with use_fourier = true: [ncoords * n_widths] float32."""
    L = lib(kind)
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    out = np.zeros(n_scores, dtype=np.float32)
    _check(L, L.lkref_fourier_scores(ctypes.byref(cfg), _p(ts_e), _p(ts_v), ts_e.size, _p(out), out.size))
    return out


def brute_fold_complex(ts_e, ts_v, freqs, segment_len, nbins, tsamp, t_ref=0.0, nthreads=1) -> np.ndarray:
    L = lib()
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    out = np.zeros((ts_e.size // segment_len, freqs.size, 2, nbins // 2 + 1), dtype=np.complex64)
    _check(L, L.lkref_brute_fold_complex(_p(ts_e), _p(ts_v), ts_e.size, _p(freqs), freqs.size, segment_len, nbins,
                                         tsamp, t_ref, nthreads, _p(out), out.size))
    return out


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


# ---- pruning leaf step ----------------------------------------------------------

PRUNE_STATS_DTYPE = np.dtype([
    ("level", np.uint64), ("seg_idx", np.uint64), ("n_branches", np.uint64), ("n_leaves", np.uint64),
    ("n_leaves_phy", np.uint64), ("n_leaves_surv", np.uint64), ("threshold", np.float32),
    ("score_min", np.float32), ("score_max", np.float32), ("pad", np.float32)])


def _check(L, rc):
    if rc != 0:
        raise RuntimeError(L.lkref_last_error().decode())


def middle_out(nsegments, ref_idx, tsegment, level):
    """(seg_idx, coord, current_coord, segment_coord) of MiddleOutScheme at a level."""
    L = lib()
    out = np.zeros(7, np.float64)
    _check(L, L.lkref_middle_out(nsegments, ref_idx, tsegment, level, _p(out)))
    return int(out[0]), (out[1], out[2]), (out[3], out[4]), (out[5], out[6])


def taylor_seed(cfg: RefCfg, n_coords: int) -> np.ndarray:
    L = lib()
    stride = (cfg.nparams + 2) * 2
    out = np.zeros(n_coords * stride, np.float64)
    n = u64()
    _check(L, L.lkref_taylor_seed(ctypes.byref(cfg), _p(out), n_coords, ctypes.byref(n)))
    return out[: n.value * stride].reshape(n.value, cfg.nparams + 2, 2)


def taylor_branch(leaves, nparams, coord_cur, nbins, eta, branch_max):
    L = lib()
    leaves = np.ascontiguousarray(leaves, np.float64)
    stride = (nparams + 2) * 2
    n = leaves.size // stride
    out = np.zeros(n * branch_max * stride, np.float64)
    org = np.zeros(n * branch_max, np.uint64)
    nout = u64()
    _check(L, L.lkref_taylor_branch(_p(leaves), n, nparams, coord_cur[0], coord_cur[1], nbins, eta,
                                    branch_max, _p(out), _p(org), ctypes.byref(nout)))
    k = nout.value
    return out[: k * stride].reshape(k, nparams + 2, 2), org[:k]


def taylor_resolve(cfg: RefCfg, leaves, coord_add, coord_cur, coord_init):
    L = lib()
    leaves = np.ascontiguousarray(leaves, np.float64)
    n = leaves.size // ((cfg.nparams + 2) * 2)
    coords = np.array([*coord_add, *coord_cur, *coord_init], np.float64)
    idx = np.zeros(n, np.uint64)
    sh = np.zeros(n, np.float32)
    _check(L, L.lkref_taylor_resolve(ctypes.byref(cfg), _p(leaves), n, _p(coords), _p(idx), _p(sh)))
    return idx, sh


def taylor_transform(leaves, indices, nparams, coord_next, coord_cur, conservative=False):
    """Returns a transformed copy of ``leaves`` (only rows named by indices change)."""
    L = lib()
    out = np.array(leaves, np.float64, copy=True, order="C")
    idx = np.ascontiguousarray(indices, np.uint64)
    ntot = out.size // ((nparams + 2) * 2)
    _check(L, L.lkref_taylor_transform(_p(out), ntot, _p(idx), idx.size, nparams, coord_next[0],
                                       coord_next[1], coord_cur[0], coord_cur[1], int(conservative)))
    return out


def shift_add_batch(folds_tree, indices_tree, folds_ffa, indices_ffa, phase_shift, nbins,
                    physical_start_idx, capacity):
    L = lib()
    ft = np.ascontiguousarray(folds_tree, np.float32)
    it = np.ascontiguousarray(indices_tree, np.uint64)
    ff = np.ascontiguousarray(folds_ffa, np.float32)
    iff = np.ascontiguousarray(indices_ffa, np.uint64)
    ps = np.ascontiguousarray(phase_shift, np.float32)
    out = np.zeros((it.size, 2, nbins), np.float32)
    _check(L, L.lkref_shift_add_batch(_p(ft), _p(it), _p(ff), _p(iff), _p(ps), _p(out), nbins, it.size,
                                      physical_start_idx, capacity))
    return out


def score_filter(folds, nbins, widths, threshold):
    L = lib()
    folds = np.ascontiguousarray(folds, np.float32)
    w = np.ascontiguousarray(widths, np.uint64)
    n = folds.size // (2 * nbins)
    scores = np.zeros(n, np.float32)
    idx = np.zeros(n, np.uint64)
    npass = u64()
    _check(L, L.lkref_score_filter(_p(folds), n, nbins, _p(w), w.size, threshold, _p(scores), _p(idx),
                                   ctypes.byref(npass)))
    return scores, idx[: npass.value]


def branching_pattern(cfg: RefCfg, ref_seg=0, conservative=False) -> np.ndarray:
    L = lib()
    out = np.zeros(4096, np.float64)
    n = u64()
    _check(L, L.lkref_branching_pattern(ctypes.byref(cfg), int(conservative), ref_seg, _p(out), out.size,
                                        ctypes.byref(n)))
    return out[: n.value].copy()


def branching_pattern_basis(cfg: RefCfg, basis="taylor", ref_seg=0, conservative=False) -> np.ndarray:
    L = lib()
    out = np.zeros(4096, np.float64)
    n = u64()
    _check(L, L.lkref_branching_pattern_basis(ctypes.byref(cfg), 1 if basis == "chebyshev" else 0,
                                              int(conservative), ref_seg, _p(out), out.size, ctypes.byref(n)))
    return out[: n.value].copy()


def taylor_to_cheby(leaves, nparams, coord_init):
    L = lib()
    out = np.array(leaves, np.float64, copy=True, order="C")
    n = out.size // ((nparams + 2) * 2)
    _check(L, L.lkref_taylor_to_cheby(_p(out), n, nparams, coord_init[0], coord_init[1]))
    return out


def cheby_to_taylor(leaves, nparams, coord_report):
    L = lib()
    out = np.array(leaves, np.float64, copy=True, order="C")
    n = out.size // ((nparams + 2) * 2)
    _check(L, L.lkref_cheby_to_taylor(_p(out), n, nparams, coord_report[0], coord_report[1]))
    return out


def cheby_branch(leaves, nparams, coord_cur, coord_prev, nbins, eta, branch_max):
    """Returns (children, origins, parents transformed to coord_cur)."""
    L = lib()
    work = np.array(leaves, np.float64, copy=True, order="C")
    stride = (nparams + 2) * 2
    n = work.size // stride
    out = np.zeros(n * branch_max * stride, np.float64)
    org = np.zeros(n * branch_max, np.uint64)
    nout = u64()
    _check(L, L.lkref_cheby_branch(_p(work), n, nparams, coord_cur[0], coord_cur[1], coord_prev[0],
                                   coord_prev[1], nbins, eta, branch_max, _p(out), _p(org), ctypes.byref(nout)))
    k = nout.value
    return out[: k * stride].reshape(k, nparams + 2, 2), org[:k], work.reshape(n, nparams + 2, 2)


def cheby_resolve(cfg: RefCfg, leaves, coord_add, coord_cur, coord_init):
    L = lib()
    leaves = np.ascontiguousarray(leaves, np.float64)
    n = leaves.size // ((cfg.nparams + 2) * 2)
    coords = np.array([*coord_add, *coord_cur, *coord_init], np.float64)
    idx = np.zeros(n, np.uint64)
    sh = np.zeros(n, np.float32)
    _check(L, L.lkref_cheby_resolve(ctypes.byref(cfg), _p(leaves), n, _p(coords), _p(idx), _p(sh)))
    return idx, sh


def cheby_transform(leaves, indices, nparams, coord_next, coord_cur):
    L = lib()
    out = np.array(leaves, np.float64, copy=True, order="C")
    idx = np.ascontiguousarray(indices, np.uint64)
    ntot = out.size // ((nparams + 2) * 2)
    _check(L, L.lkref_cheby_transform(_p(out), ntot, _p(idx), idx.size, nparams, coord_next[0], coord_next[1],
                                      coord_cur[0], coord_cur[1]))
    return out


def branch_max(cfg: RefCfg, conservative=False) -> int:
    L = lib()
    out = u64()
    _check(L, L.lkref_branch_max(ctypes.byref(cfg), int(conservative), ctypes.byref(out)))
    return out.value


def prune_run(cfg: RefCfg, ffa_fold, thresholds, ref_seg, max_sugg, batch_size, branch_max_,
              n_iters, nbins, conservative=False, kind="parity", basis="taylor"):
    """One reference pruning run: returns (stats, leaves, folds, scores) of the final tree."""
    L = lib(kind)
    ffa = np.ascontiguousarray(ffa_fold, np.float32).ravel()
    thr = np.ascontiguousarray(thresholds, np.float32)
    stats = np.zeros(n_iters + 1, PRUNE_STATS_DTYPE)
    nstats = u64()
    stride = (cfg.nparams + 2) * 2
    leaves = np.zeros(max_sugg * stride, np.float64)
    folds = np.zeros(max_sugg * 2 * nbins, np.float32)
    scores = np.zeros(max_sugg, np.float32)
    n = u64()
    _check(L, L.lkref_prune_run_basis(1 if basis == "chebyshev" else 0, ctypes.byref(cfg), int(conservative),
                                      _p(ffa), ffa.size, _p(thr), thr.size, ref_seg, max_sugg, batch_size,
                                      branch_max_, n_iters, _p(stats), ctypes.byref(nstats), _p(leaves),
                                      _p(folds), _p(scores), max_sugg, ctypes.byref(n)))
    k = n.value
    return (stats[: nstats.value], leaves[: k * stride].reshape(k, cfg.nparams + 2, 2),
            folds[: k * 2 * nbins].reshape(k, 2, nbins), scores[:k])


def snr_threshold(profiles, nbins, widths, thresholds, stdnoise) -> np.ndarray:
    """snr_boxcar_threshold_with_cache per profile (bool array)."""
    L = lib()
    p = np.ascontiguousarray(profiles, np.float32)
    n = p.size // nbins
    w = np.ascontiguousarray(widths, np.uint64)
    t = np.ascontiguousarray(np.broadcast_to(np.asarray(thresholds, np.float32), (n,)))
    out = np.zeros(n, np.uint8)
    _check(L, L.lkref_snr_threshold(_p(p), n, nbins, _p(w), w.size, _p(t), stdnoise, _p(out)))
    return out.astype(bool)


def region_plan(cfg: RefCfg, max_memory_gb=8.0, octave_scale=2.0, nbins_max=1024, max_passing=1 << 22,
                use_gpu=False, complex_fold=None, use_fourier=False):
    """FFARegionPlanner<float> of the reference: (chunks [n, 6] = f_min, f_max,
    nbins, eta, bseg_brute, bseg_ffa; stats [5] = max buffer size, max coord
    size, max ncoords, max levels, sweep memory usage in GB -- the device
    model when use_gpu)."""
    L = lib()
    cap = 4096
    rows = np.zeros(cap * 6, np.float64)
    stats = np.zeros(5, np.float64)
    n = u64()
    if complex_fold is None and not use_fourier:
        _check(L, L.lkref_region_plan(ctypes.byref(cfg), max_memory_gb, octave_scale, nbins_max, max_passing,
                                      int(use_gpu), _p(rows), cap, ctypes.byref(n), _p(stats)))
    else:
        cf = bool(use_fourier) if complex_fold is None else bool(complex_fold)
        _check(L, L.lkref_region_plan_typed(ctypes.byref(cfg), max_memory_gb, octave_scale, nbins_max, max_passing,
                                            int(use_gpu), int(cf), int(bool(use_fourier)), _p(rows), cap,
                                            ctypes.byref(n), _p(stats)))
    k = min(n.value, cap)
    return rows[: k * 6].reshape(k, 6), stats


def prune_run_full(cfg: RefCfg, ffa_fold, thresholds, ref_seg, max_sugg, batch_size, branch_max_, n_iters,
                   nbins, conservative=False, basis="taylor"):
    """A whole reference pruning run with the survivors ascended and reported:
    (stats, leaves, folds, scores, scores_ep)."""
    L = lib()
    ffa = np.ascontiguousarray(ffa_fold, np.float32).ravel()
    thr = np.ascontiguousarray(thresholds, np.float32)
    stats = np.zeros(n_iters + 1, PRUNE_STATS_DTYPE)
    nstats = u64()
    stride = (cfg.nparams + 2) * 2
    leaves = np.zeros(max_sugg * stride, np.float64)
    folds = np.zeros(max_sugg * 2 * nbins, np.float32)
    scores = np.zeros(max_sugg, np.float32)
    scores_ep = np.zeros(max_sugg, np.float32)
    n = u64()
    _check(L, L.lkref_prune_run_full(1 if basis == "chebyshev" else 0, ctypes.byref(cfg), int(conservative),
                                     _p(ffa), ffa.size, _p(thr), thr.size, ref_seg, max_sugg, batch_size,
                                     branch_max_, n_iters, _p(stats), ctypes.byref(nstats), _p(leaves),
                                     _p(folds), _p(scores), _p(scores_ep), max_sugg, ctypes.byref(n)))
    k = n.value
    return (stats[: nstats.value], leaves[: k * stride].reshape(k, cfg.nparams + 2, 2),
            folds[: k * 2 * nbins].reshape(k, 2, nbins), scores[:k], scores_ep[:k])


# ---- DynamicThresholdScheme pieces (lib/scheme.cpp, lib/simulation.cpp,
# lib/utils.cpp, thresholds.hpp) and the restated stage loop -----------------

def _chk(L, rc):
    if rc != 0:
        raise RuntimeError(L.lkref_last_error().decode())


def dts_thresholds(snr_start, snr_final, n, kind="parity"):
    L = lib(kind)
    out = np.zeros(n, np.float32)
    _chk(L, L.lkref_dts_thresholds(snr_start, snr_final, n, _p(out)))
    return out


def dts_probs(n, prob_min, kind="parity"):
    L = lib(kind)
    out = np.zeros(n, np.float32)
    _chk(L, L.lkref_dts_probs(n, prob_min, _p(out)))
    return out


def dts_profile(nbins, ducy, center=0.5, kind="parity"):
    L = lib(kind)
    out = np.zeros(nbins, np.float32)
    _chk(L, L.lkref_dts_profile(nbins, ducy, center, _p(out)))
    return out


def dts_bound(nstages, snr_bound, kind="parity"):
    L = lib(kind)
    out = np.zeros(nstages, np.float32)
    _chk(L, L.lkref_dts_bound(nstages, snr_bound, _p(out)))
    return out


def dts_neighbours(indices, target, num, kind="parity"):
    L = lib(kind)
    idx = np.ascontiguousarray(indices, np.uint64)
    out = np.zeros(max(1, idx.size), np.uint64)
    n = u64()
    _chk(L, L.lkref_dts_neighbours(_p(idx), idx.size, target, num, _p(out), ctypes.byref(n)))
    return out[: n.value].copy()


def dts_lower_bin(range_, value, kind="parity"):
    r = np.ascontiguousarray(range_, np.float32)
    return int(lib(kind).lkref_dts_lower_bin(_p(r), r.size, value))


def dts_gen_next(state, threshold, s0, s1, nbranches, dtype, kind="parity"):
    L = lib(kind)
    st = np.ascontiguousarray(np.asarray([state], dtype=dtype))
    out = np.zeros(1, dtype)
    _chk(L, L.lkref_dts_gen_next(_p(st), threshold, s0, s1, nbranches, _p(out)))
    return out[0]


def dts_best_path(states, nstages, thresholds, probs, min_pd=0.1, kind="parity"):
    L = lib(kind)
    st = np.ascontiguousarray(states)
    th = np.ascontiguousarray(thresholds, np.float32)
    pr = np.ascontiguousarray(probs, np.float32)
    out = np.zeros(nstages, np.float32)
    n = u64()
    _chk(L, L.lkref_dts_best_path(_p(st), nstages, _p(th), th.size, _p(pr), pr.size, min_pd, _p(out),
                                  ctypes.byref(n)))
    return out[: n.value].copy()


def dts_run(branching, ref_ducy, guess, lut, dtype, nbins=64, ntrials=1024, nprobs=10, prob_min=0.05, snr_final=8.0,
            nthresholds=100, ducy_max=0.3, wtsp=1.0, beam_width=0.7, seed=0x10C1B200, thres_neigh=10,
            stages_run=0, kind="parity"):
    L = lib(kind)
    b = np.ascontiguousarray(branching, np.float32)
    g = np.ascontiguousarray(guess, np.float32)
    lt = np.ascontiguousarray(lut, np.float32)
    out = np.zeros(b.size * nthresholds * nprobs, dtype)
    _chk(L, L.lkref_dts_run(_p(b), b.size, ref_ducy, nbins, ntrials, nprobs, prob_min, snr_final, nthresholds,
                            ducy_max, wtsp, beam_width, seed, thres_neigh, _p(g), _p(lt), stages_run, _p(out)))
    return out
