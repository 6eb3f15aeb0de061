"""ctypes binding of the C oracle (``oracle/loki_oracle.c``). Test infrastructure only."""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

MAX_LEVELS = 40
MAX_PARAMS = 5
MAX_WIDTHS = 64

u64 = ctypes.c_uint64
u32 = ctypes.c_uint32
f64 = ctypes.c_double
f32 = ctypes.c_float
vp = ctypes.c_void_p


class Cfg(ctypes.Structure):
    _fields_ = [
        ("nsamps", u64),
        ("tsamp", f64),
        ("nbins", u64),
        ("eta", f64),
        ("nparams", u32),
        ("limits", f64 * (2 * MAX_PARAMS)),
        ("bseg_brute", u64),
        ("bseg_ffa", u64),
        ("ducy_max", f64),
        ("wtsp", f64),
    ]


class Plan(ctypes.Structure):
    _fields_ = [
        ("nparams", u32),
        ("n_levels", u32),
        ("nsamps", u64),
        ("nbins", u64),
        ("tsamp", f64),
        ("eta", f64),
        ("tseg_brute", f64),
        ("bseg_brute", u64),
        ("bseg_ffa", u64),
        ("limits", f64 * (2 * MAX_PARAMS)),
        ("segment_lens", u64 * MAX_LEVELS),
        ("nsegments", u64 * MAX_LEVELS),
        ("tsegments", f64 * MAX_LEVELS),
        ("ncoords", u64 * MAX_LEVELS),
        ("ncoords_offsets", u32 * (MAX_LEVELS + 1)),
        ("param_counts", (u64 * MAX_PARAMS) * MAX_LEVELS),
        ("dparams", (f64 * MAX_PARAMS) * MAX_LEVELS),
        ("buffer_size", u64),
        ("coord_size", u64),
        ("n_widths", u32),
        ("widths", u64 * MAX_WIDTHS),
    ]


COORD_FREQ_DTYPE = np.dtype([("idx", np.uint32), ("shift", np.float32)])
COORD_DTYPE = np.dtype(
    [("i_tail", np.uint32), ("shift_tail", np.float32), ("i_head", np.uint32), ("shift_head", np.float32)]
)

_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"oracle library missing: {_LIB_PATH} (run `make -C oracle oracle`)")
        L = ctypes.CDLL(_LIB_PATH)
        L.lko_last_error.restype = ctypes.c_char_p
        L.lko_plan_create.argtypes = [vp, vp]
        L.lko_resolve_freq.argtypes = [vp, vp]
        L.lko_resolve_taylor.argtypes = [vp, vp]
        L.lko_phase_idx.restype = f32
        L.lko_phase_idx.argtypes = [f64, f64, u64, f64]
        L.lko_phase_idx_uint.restype = u32
        L.lko_phase_idx_uint.argtypes = [f64, f64, u64, f64]
        L.lko_param_val_at_idx.restype = f64
        L.lko_param_val_at_idx.argtypes = [f64, f64, u64, u64]
        L.lko_nearest_idx.restype = u64
        L.lko_nearest_idx.argtypes = [f64, f64, f64, u64]
        L.lko_range_param.restype = u64
        L.lko_range_param.argtypes = [f64, f64, f64, vp, u64]
        L.lko_box_widths.restype = u64
        L.lko_box_widths.argtypes = [u64, f64, f64, vp, u64]
        L.lko_brute_fold.argtypes = [vp, vp, u64, vp, u64, u64, u64, f64, f64, vp]
        L.lko_phase_map.argtypes = [vp, u64, u64, u64, f64, f64, vp]
        L.lko_merge_freq.argtypes = [vp, vp, vp, u64, u64, u64, u64]
        L.lko_merge_taylor.argtypes = [vp, vp, vp, u64, u64, u64, u64]
        L.lko_ffa.argtypes = [vp, vp, vp, u32, vp]
        L.lko_ffa_scores64.argtypes = [vp, vp, vp, vp, u64, vp]
        L.lko_snr_boxcar_3d.argtypes = [vp, u64, u64, vp, u64, vp]
        L.lko_snr_boxcar_3d_max.argtypes = [vp, u64, u64, vp, u64, vp]
        L.lko_snr_boxcar_2d_max.argtypes = [vp, u64, u64, vp, u64, f32, vp]
        L.lko_circular_prefix_sum.argtypes = [vp, vp, u64, u64]
        L.lko_compact.restype = u64
        L.lko_compact.argtypes = [vp, u64, f32, vp, vp]
        L.lko_middle_out.argtypes = [u64, u64, f64, u64, vp]
        L.lko_taylor_seed.restype = u64
        L.lko_taylor_seed.argtypes = [vp, vp]
        L.lko_taylor_branch.argtypes = [vp, u64, u32, f64, f64, u64, f64, u64, vp, vp, u64, vp]
        L.lko_taylor_resolve.argtypes = [vp, vp, u64, vp, vp, vp]
        L.lko_taylor_transform.argtypes = [vp, vp, u64, u32, f64, f64, ctypes.c_int]
        L.lko_shift_add_batch.argtypes = [vp, vp, vp, vp, vp, vp, u64, u64, u64, u64]
        L.lko_score_filter.restype = u64
        L.lko_score_filter.argtypes = [vp, u64, u64, vp, u64, f32, vp, vp]
        L.lko_snr_max_div.restype = f32
        L.lko_snr_max_div.argtypes = [vp, u64, vp, u64, f32]
        L.lko_mc_stage.restype = u64
        L.lko_mc_stage.argtypes = [vp, vp, u64, u64, vp, vp, ctypes.c_int, f32, vp, f32, f32, vp, u64, f32, vp,
                                   u64, vp, vp, vp, vp, vp]
        L.lko_prune_run.argtypes = [vp, ctypes.c_int, vp, vp, u64, u64, u64, u64, u64, u64, vp, vp,
                                    vp, vp, vp, u64, vp]
        L.lko_prune_finalize.argtypes = [vp, ctypes.c_int, vp, u64, u64, vp, vp, vp, vp, u64]
        L.lko_prune_run_basis.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, u64, u64, u64, u64, u64,
                                          u64, vp, vp, vp, vp, vp, u64, vp]
        L.lko_taylor_to_cheby.argtypes = [vp, u64, u32, f64]
        L.lko_cheby_to_taylor.argtypes = [vp, u64, u32, f64]
        L.lko_cheby_transform.argtypes = [vp, vp, u64, u32, f64, f64, f64, f64]
        L.lko_cheby_branch.argtypes = [vp, u64, u32, f64, f64, f64, f64, u64, f64, u64, vp, vp, u64, vp]
        L.lko_cheby_resolve.argtypes = [vp, vp, u64, vp, vp, vp]
        L.lko_fourier_brute_fold.argtypes = [vp, vp, u64, vp, u64, u64, u64, f64, f64, vp]
        L.lko_fourier_merge.argtypes = [vp, vp, vp, ctypes.c_int, u64, u64, u64, u64]
        L.lko_irfft.argtypes = [vp, vp, u64, u64]
        L.lko_rfft.argtypes = [vp, vp, u64, u64]
        L.lko_ffa_fourier.argtypes = [vp, vp, vp, u32, u64, vp]
        L.lko_ffa_fourier_scores64.argtypes = [vp, vp, vp, u64, vp, u64, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(lib().lko_last_error().decode())


def make_cfg(
    nsamps: int,
    tsamp: float,
    nbins: int,
    eta: float,
    param_limits,
    bseg_brute: int | None = None,
    bseg_ffa: int | None = None,
    ducy_max: float = 0.2,
    wtsp: float = 1.5,
) -> Cfg:
    lim = np.asarray(param_limits, dtype=np.float64).reshape(-1, 2)
    c = Cfg()
    c.nsamps = nsamps
    c.tsamp = tsamp
    c.nbins = nbins
    c.eta = eta
    c.nparams = lim.shape[0]
    for i, (a, b) in enumerate(lim):
        c.limits[2 * i] = a
        c.limits[2 * i + 1] = b
    c.bseg_brute = bseg_brute or 0
    c.bseg_ffa = bseg_ffa or 0
    c.ducy_max = ducy_max
    c.wtsp = wtsp
    return c


@dataclass
class OraclePlan:
    raw: Plan

    @property
    def n_levels(self) -> int:
        return self.raw.n_levels

    @property
    def nparams(self) -> int:
        return self.raw.nparams

    @property
    def nbins(self) -> int:
        return self.raw.nbins

    @property
    def ncoords(self) -> np.ndarray:
        return np.array(self.raw.ncoords[: self.n_levels], dtype=np.uint64)

    @property
    def nsegments(self) -> np.ndarray:
        return np.array(self.raw.nsegments[: self.n_levels], dtype=np.uint64)

    @property
    def segment_lens(self) -> np.ndarray:
        return np.array(self.raw.segment_lens[: self.n_levels], dtype=np.uint64)

    @property
    def ncoords_offsets(self) -> np.ndarray:
        return np.array(self.raw.ncoords_offsets[: self.n_levels + 1], dtype=np.uint32)

    @property
    def param_counts(self) -> np.ndarray:
        return np.array([list(self.raw.param_counts[l][: self.nparams]) for l in range(self.n_levels)], dtype=np.uint64)

    @property
    def dparams(self) -> np.ndarray:
        return np.array([list(self.raw.dparams[l][: self.nparams]) for l in range(self.n_levels)])

    @property
    def widths(self) -> np.ndarray:
        return np.array(self.raw.widths[: self.raw.n_widths], dtype=np.uint64)

    @property
    def buffer_size(self) -> int:
        return self.raw.buffer_size

    @property
    def coord_size(self) -> int:
        return self.raw.coord_size

    def fold_size(self, level: int | None = None) -> int:
        l = self.n_levels - 1 if level is None else level
        return int(self.nsegments[l] * self.ncoords[l] * 2 * self.nbins)

    def freqs0(self) -> np.ndarray:
        r = self.raw
        np_ = self.nparams
        n = int(r.param_counts[0][np_ - 1])
        out = np.zeros(n, dtype=np.float64)
        lib().lko_range_param(r.limits[2 * (np_ - 1)], r.limits[2 * (np_ - 1) + 1], r.dparams[0][np_ - 1], _p(out), n)
        return out

    def t_ref0(self) -> float:
        return 0.0 if self.nparams == 1 else self.raw.tsegments[0] / 2.0


def plan_create(cfg: Cfg) -> OraclePlan:
    p = Plan()
    _check(lib().lko_plan_create(ctypes.byref(cfg), ctypes.byref(p)))
    return OraclePlan(p)


def resolve(plan: OraclePlan) -> np.ndarray:
    if plan.nparams == 1:
        out = np.zeros(plan.coord_size, dtype=COORD_FREQ_DTYPE)
        _check(lib().lko_resolve_freq(ctypes.byref(plan.raw), _p(out)))
    else:
        out = np.zeros(plan.coord_size, dtype=COORD_DTYPE)
        _check(lib().lko_resolve_taylor(ctypes.byref(plan.raw), _p(out)))
    return out


def brute_fold(ts_e, ts_v, freqs, segment_len, nbins, tsamp, t_ref=0.0) -> np.ndarray:
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    nseg = ts_e.size // segment_len
    out = np.zeros(nseg * freqs.size * 2 * nbins, dtype=np.float32)
    _check(lib().lko_brute_fold(_p(ts_e), _p(ts_v), ts_e.size, _p(freqs), freqs.size, segment_len, nbins, tsamp, t_ref, _p(out)))
    return out


def phase_map(freqs, segment_len, nbins, tsamp, t_ref=0.0) -> np.ndarray:
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    out = np.zeros((freqs.size, segment_len), dtype=np.uint32)
    lib().lko_phase_map(_p(freqs), freqs.size, segment_len, nbins, tsamp, t_ref, _p(out))
    return out


def ffa(plan: OraclePlan, ts_e, ts_v, level: int | None = None) -> np.ndarray:
    l = plan.n_levels - 1 if level is None else level
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    out = np.zeros(plan.fold_size(l), dtype=np.float32)
    _check(lib().lko_ffa(ctypes.byref(plan.raw), _p(ts_e), _p(ts_v), l, _p(out)))
    return out


def ffa_scores64(plan: OraclePlan, ts_e, ts_v, widths) -> np.ndarray:
    """FP64 FFA + boxcar S/N of every final cell and width, [ncoords, nwidths]
    float64 (the FP32 path's phase map, coordinates and shifts; every sum in
    double)."""
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    w = np.ascontiguousarray(widths, dtype=np.uint64)
    out = np.zeros((int(plan.ncoords[-1]), w.size), dtype=np.float64)
    _check(lib().lko_ffa_scores64(ctypes.byref(plan.raw), _p(ts_e), _p(ts_v), _p(w), w.size, _p(out)))
    return out


# Fourier-domain FFA (FFA<ComplexType>), every sum in double. Complex
# results are complex128 arrays; folds [nseg, ncoords, 2, nbins // 2 + 1].
NBINS_MIN_LOSSY = 64  # PulsarSearchConfig's nbins_min_lossy_bf default


def fourier_brute_fold(ts_e, ts_v, freqs, segment_len, nbins, tsamp, t_ref=0.0) -> np.ndarray:
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    freqs = np.ascontiguousarray(freqs, dtype=np.float64)
    nseg = ts_e.size // segment_len
    nbf = nbins // 2 + 1
    out = np.zeros((nseg, freqs.size, 2, nbf), dtype=np.complex128)
    _check(lib().lko_fourier_brute_fold(_p(ts_e), _p(ts_v), ts_e.size, _p(freqs), freqs.size, segment_len, nbins,
                                        tsamp, t_ref, _p(out)))
    return out


def fourier_merge(fold_in, coords, ncur, nprev, nseg, nbins) -> np.ndarray:
    fold_in = np.ascontiguousarray(fold_in, dtype=np.complex128)
    coords = np.ascontiguousarray(coords)
    taylor = 1 if coords.dtype == COORD_DTYPE else 0
    out = np.zeros((nseg, ncur, 2, nbins // 2 + 1), dtype=np.complex128)
    lib().lko_fourier_merge(_p(fold_in), _p(out), _p(coords), taylor, ncur, nprev, nseg, nbins)
    return out


def irfft(x, n) -> np.ndarray:
    """Inverse real transforms of size n over the profiles of x (its last
    axis the n // 2 + 1 harmonics, or flat): [..., n] float64."""
    nbf = n // 2 + 1
    x = np.ascontiguousarray(x, dtype=np.complex128)
    if x.size % nbf != 0:
        raise ValueError("irfft: input size is not a multiple of n // 2 + 1")
    nprof = x.size // nbf
    shape = x.shape[:-1] + (n,) if x.ndim > 1 and x.shape[-1] == nbf else (nprof * n,)
    out = np.zeros(nprof * n, dtype=np.float64)
    lib().lko_irfft(_p(x), _p(out), nprof, n)
    return out.reshape(shape)


def rfft(x, n) -> np.ndarray:
    """Real transforms of size n over the profiles of x (its last axis n, or
    flat): [..., n // 2 + 1] complex128."""
    nbf = n // 2 + 1
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.size % n != 0:
        raise ValueError("rfft: input size is not a multiple of n")
    nprof = x.size // n
    shape = x.shape[:-1] + (nbf,) if x.ndim > 1 and x.shape[-1] == n else (nprof * nbf,)
    out = np.zeros(nprof * nbf, dtype=np.complex128)
    lib().lko_rfft(_p(x), _p(out), nprof, n)
    return out.reshape(shape)


def ffa_fourier(plan: OraclePlan, ts_e, ts_v, level: int | None = None,
                nbins_min_lossy: int = NBINS_MIN_LOSSY) -> np.ndarray:
    l = plan.n_levels - 1 if level is None else level
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    nbf = plan.nbins // 2 + 1
    out = np.zeros((int(plan.nsegments[l]), int(plan.ncoords[l]), 2, nbf), dtype=np.complex128)
    _check(lib().lko_ffa_fourier(ctypes.byref(plan.raw), _p(ts_e), _p(ts_v), l, nbins_min_lossy, _p(out)))
    return out


def ffa_fourier_scores64(plan: OraclePlan, ts_e, ts_v, widths,
                         nbins_min_lossy: int = NBINS_MIN_LOSSY) -> np.ndarray:
    ts_e = np.ascontiguousarray(ts_e, dtype=np.float32)
    ts_v = np.ascontiguousarray(ts_v, dtype=np.float32)
    w = np.ascontiguousarray(widths, dtype=np.uint64)
    out = np.zeros((int(plan.ncoords[-1]), w.size), dtype=np.float64)
    _check(lib().lko_ffa_fourier_scores64(ctypes.byref(plan.raw), _p(ts_e), _p(ts_v), nbins_min_lossy, _p(w),
                                          w.size, _p(out)))
    return out


def snr_boxcar_3d(folds, widths, nbins) -> np.ndarray:
    folds = np.ascontiguousarray(folds, dtype=np.float32)
    w = np.ascontiguousarray(widths, dtype=np.uint64)
    nprof = folds.size // (2 * nbins)
    out = np.zeros((nprof, w.size), dtype=np.float32)
    lib().lko_snr_boxcar_3d(_p(folds), nprof, nbins, _p(w), w.size, _p(out))
    return out


def snr_boxcar_3d_max(folds, widths, nbins) -> np.ndarray:
    folds = np.ascontiguousarray(folds, dtype=np.float32)
    w = np.ascontiguousarray(widths, dtype=np.uint64)
    nprof = folds.size // (2 * nbins)
    out = np.zeros(nprof, dtype=np.float32)
    lib().lko_snr_boxcar_3d_max(_p(folds), nprof, nbins, _p(w), w.size, _p(out))
    return out


def snr_boxcar_2d_max(folds, widths, nbins, stdnoise=1.0) -> np.ndarray:
    folds = np.ascontiguousarray(folds, dtype=np.float32)
    w = np.ascontiguousarray(widths, dtype=np.uint64)
    nprof = folds.size // nbins
    out = np.zeros(nprof, dtype=np.float32)
    lib().lko_snr_boxcar_2d_max(_p(folds), nprof, nbins, _p(w), w.size, stdnoise, _p(out))
    return out


def circular_prefix_sum(x, nsum) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    # The reference always writes the first nbins entries, even when nsum < nbins.
    out = np.zeros(max(nsum, x.size), dtype=np.float32)
    lib().lko_circular_prefix_sum(_p(x), _p(out), x.size, nsum)
    return out[:nsum].copy()


def merge_freq(fold_in, coords, ncur, nprev, nseg, nbins) -> np.ndarray:
    fold_in = np.ascontiguousarray(fold_in, dtype=np.float32)
    coords = np.ascontiguousarray(coords, dtype=COORD_FREQ_DTYPE)
    out = np.zeros(nseg * ncur * 2 * nbins, dtype=np.float32)
    lib().lko_merge_freq(_p(fold_in), _p(out), _p(coords), ncur, nprev, nseg, nbins)
    return out


def merge_taylor(fold_in, coords, ncur, nprev, nseg, nbins) -> np.ndarray:
    fold_in = np.ascontiguousarray(fold_in, dtype=np.float32)
    coords = np.ascontiguousarray(coords, dtype=COORD_DTYPE)
    out = np.zeros(nseg * ncur * 2 * nbins, dtype=np.float32)
    lib().lko_merge_taylor(_p(fold_in), _p(out), _p(coords), ncur, nprev, nseg, nbins)
    return out


def compact(scores, snr_min) -> tuple[np.ndarray, np.ndarray]:
    s = np.ascontiguousarray(scores, dtype=np.float32).ravel()
    idx = np.zeros(s.size, dtype=np.uint32)
    val = np.zeros(s.size, dtype=np.float32)
    n = lib().lko_compact(_p(s), s.size, snr_min, _p(idx), _p(val))
    return idx[:n].copy(), val[:n].copy()


def box_widths(nbins, ducy_max=0.2, wtsp=1.5) -> np.ndarray:
    out = np.zeros(MAX_WIDTHS, dtype=np.uint64)
    n = lib().lko_box_widths(nbins, ducy_max, wtsp, _p(out), MAX_WIDTHS)
    return out[:n].copy()


def phase_idx(t, f, nbins, delay=0.0) -> float:
    return lib().lko_phase_idx(t, f, nbins, delay)


def phase_idx_uint(t, f, nbins, delay=0.0) -> int:
    return lib().lko_phase_idx_uint(t, f, nbins, delay)


def nearest_idx(val, vmin, vmax, count) -> int:
    return lib().lko_nearest_idx(val, vmin, vmax, count)


def param_val_at_idx(vmin, vmax, count, i) -> float:
    return lib().lko_param_val_at_idx(vmin, vmax, count, i)


# ---- pruning leaf step ----------------------------------------------------------

PRUNE_STATS_DTYPE = np.dtype([
    ("level", np.uint64), ("seg_idx", np.uint64), ("n_branches", np.uint64), ("n_leaves", np.uint64),
    ("n_leaves_phy", np.uint64), ("n_leaves_surv", np.uint64), ("threshold", np.float32),
    ("score_min", np.float32), ("score_max", np.float32), ("pad", np.float32)])


def middle_out(nsegments, ref_idx, tsegment, level):
    """(seg_idx, coord, current_coord, segment_coord) of MiddleOutScheme at a level."""
    out = np.zeros(7, np.float64)
    _check(lib().lko_middle_out(nsegments, ref_idx, tsegment, level, _p(out)))
    return int(out[0]), (out[1], out[2]), (out[3], out[4]), (out[5], out[6])


def taylor_seed(plan: OraclePlan) -> np.ndarray:
    np_ = plan.nparams
    n = int(plan.ncoords[-1])
    out = np.zeros((n, np_ + 2, 2), np.float64)
    k = lib().lko_taylor_seed(ctypes.byref(plan.raw), _p(out))
    if k != n:
        raise RuntimeError(lib().lko_last_error().decode())
    return out


def taylor_branch(leaves, nparams, coord_cur, nbins, eta, branch_max, cap=None):
    leaves = np.ascontiguousarray(leaves, np.float64)
    stride = (nparams + 2) * 2
    n = leaves.size // stride
    cap = n * branch_max if cap is None else cap
    out = np.zeros(cap * stride, np.float64)
    org = np.zeros(cap, np.uint64)
    nout = u64()
    rc = lib().lko_taylor_branch(_p(leaves), n, nparams, coord_cur[0], coord_cur[1], nbins, eta, branch_max,
                                 _p(out), _p(org), cap, ctypes.byref(nout))
    if rc == 2:
        return taylor_branch(leaves, nparams, coord_cur, nbins, eta, branch_max, cap=nout.value)
    _check(rc)
    k = nout.value
    return out[: k * stride].reshape(k, nparams + 2, 2), org[:k]


def taylor_resolve(plan: OraclePlan, leaves, coord_add, coord_cur, coord_init):
    leaves = np.ascontiguousarray(leaves, np.float64)
    n = leaves.size // ((plan.nparams + 2) * 2)
    coords = np.array([*coord_add, *coord_cur, *coord_init], np.float64)
    idx = np.zeros(n, np.uint64)
    sh = np.zeros(n, np.float32)
    lib().lko_taylor_resolve(ctypes.byref(plan.raw), _p(leaves), n, _p(coords), _p(idx), _p(sh))
    return idx, sh


def taylor_transform(leaves, indices, nparams, coord_next, coord_cur, conservative=False):
    out = np.array(leaves, np.float64, copy=True, order="C")
    idx = np.ascontiguousarray(indices, np.uint64)
    lib().lko_taylor_transform(_p(out), _p(idx), idx.size, nparams, coord_next[0], coord_cur[0],
                               int(conservative))
    return out


def shift_add_batch(folds_tree, indices_tree, folds_ffa, indices_ffa, phase_shift, nbins,
                    physical_start_idx, capacity):
    ft = np.ascontiguousarray(folds_tree, np.float32)
    it = np.ascontiguousarray(indices_tree, np.uint64)
    ff = np.ascontiguousarray(folds_ffa, np.float32)
    iff = np.ascontiguousarray(indices_ffa, np.uint64)
    ps = np.ascontiguousarray(phase_shift, np.float32)
    out = np.zeros((it.size, 2, nbins), np.float32)
    lib().lko_shift_add_batch(_p(ft), _p(it), _p(ff), _p(iff), _p(ps), _p(out), nbins, it.size,
                              physical_start_idx, capacity)
    return out


def score_filter(folds, nbins, widths, threshold):
    folds = np.ascontiguousarray(folds, np.float32)
    w = np.ascontiguousarray(widths, np.uint64)
    n = folds.size // (2 * nbins)
    scores = np.zeros(n, np.float32)
    idx = np.zeros(n, np.uint64)
    k = lib().lko_score_filter(_p(folds), n, nbins, _p(w), w.size, threshold, _p(scores), _p(idx))
    return scores, idx[:k]


# ---- Chebyshev basis (lib/chebyshev.cpp) --------------------------------------

def taylor_to_cheby(leaves, nparams, coord_init):
    out = np.array(leaves, np.float64, copy=True, order="C")
    n = out.size // ((nparams + 2) * 2)
    lib().lko_taylor_to_cheby(_p(out), n, nparams, coord_init[1])
    return out


def cheby_to_taylor(leaves, nparams, coord_report):
    out = np.array(leaves, np.float64, copy=True, order="C")
    n = out.size // ((nparams + 2) * 2)
    lib().lko_cheby_to_taylor(_p(out), n, nparams, coord_report[1])
    return out


def cheby_transform(leaves, indices, nparams, coord_next, coord_cur):
    out = np.array(leaves, np.float64, copy=True, order="C")
    idx = np.ascontiguousarray(indices, np.uint64)
    lib().lko_cheby_transform(_p(out), _p(idx), idx.size, nparams, coord_next[0], coord_next[1],
                              coord_cur[0], coord_cur[1])
    return out


def cheby_branch(leaves, nparams, coord_cur, coord_prev, nbins, eta, branch_max, cap=None):
    """Returns (children, origins, parents transformed to coord_cur)."""
    par = np.array(leaves, np.float64, copy=True, order="C")
    stride = (nparams + 2) * 2
    n = par.size // stride
    cap = n * branch_max if cap is None else cap
    out = np.zeros(cap * stride, np.float64)
    org = np.zeros(cap, np.uint64)
    nout = u64()
    work = par.copy()
    rc = lib().lko_cheby_branch(_p(work), n, nparams, coord_cur[0], coord_cur[1], coord_prev[0], coord_prev[1],
                                nbins, eta, branch_max, _p(out), _p(org), cap, ctypes.byref(nout))
    if rc == 2:
        return cheby_branch(leaves, nparams, coord_cur, coord_prev, nbins, eta, branch_max, cap=nout.value)
    _check(rc)
    k = nout.value
    return out[: k * stride].reshape(k, nparams + 2, 2), org[:k], work.reshape(n, nparams + 2, 2)


def cheby_resolve(plan: OraclePlan, leaves, coord_add, coord_cur, coord_init):
    leaves = np.ascontiguousarray(leaves, np.float64)
    n = leaves.size // ((plan.nparams + 2) * 2)
    coords = np.array([*coord_add, *coord_cur, *coord_init], np.float64)
    idx = np.zeros(n, np.uint64)
    sh = np.zeros(n, np.float32)
    lib().lko_cheby_resolve(ctypes.byref(plan.raw), _p(leaves), n, _p(coords), _p(idx), _p(sh))
    return idx, sh


def prune_run(plan: OraclePlan, ffa_fold, thresholds, ref_seg, max_sugg, batch_size, branch_max,
              n_iters, conservative=False, basis="taylor"):
    """One pruning run: returns (stats, leaves, folds, scores) of the final tree."""
    ffa = np.ascontiguousarray(ffa_fold, np.float32).ravel()
    thr = np.ascontiguousarray(thresholds, np.float32)
    nbins = plan.nbins
    stats = np.zeros(n_iters + 1, PRUNE_STATS_DTYPE)
    nstats = u64()
    stride = (plan.nparams + 2) * 2
    leaves = np.zeros(max_sugg * stride, np.float64)
    folds = np.zeros(max_sugg * 2 * nbins, np.float32)
    scores = np.zeros(max_sugg, np.float32)
    n = u64()
    _check(lib().lko_prune_run_basis(ctypes.byref(plan.raw), 1 if basis == "chebyshev" else 0, int(conservative),
                                     _p(ffa), _p(thr), thr.size, ref_seg, max_sugg, batch_size, branch_max,
                                     n_iters, _p(stats), ctypes.byref(nstats), _p(leaves), _p(folds), _p(scores),
                                     max_sugg, ctypes.byref(n)))
    k = n.value
    return (stats[: nstats.value], leaves[: k * stride].reshape(k, plan.nparams + 2, 2),
            folds[: k * 2 * nbins].reshape(k, 2, nbins), scores[:k])


def prune_finalize(plan: OraclePlan, ffa_fold, ref_seg, prune_level, leaves, folds, scores, basis="taylor"):
    """Ascend + report of a run's survivors (copies): returns (leaves, folds,
    scores, scores_ep)."""
    ffa = np.ascontiguousarray(ffa_fold, np.float32).ravel()
    lv = np.ascontiguousarray(leaves, np.float64).copy()
    fo = np.ascontiguousarray(folds, np.float32).copy()
    sc = np.ascontiguousarray(scores, np.float32).copy()
    ep = np.zeros_like(sc)
    _check(lib().lko_prune_finalize(ctypes.byref(plan.raw), 1 if basis == "chebyshev" else 0, _p(ffa), ref_seg,
                                    prune_level, _p(lv), _p(fo), _p(sc), _p(ep), sc.size))
    return lv, fo, sc, ep


# ---- Monte-Carlo threshold stage -------------------------------------------------

def snr_max_div(profiles, nbins, widths, stdnoise) -> np.ndarray:
    p = np.ascontiguousarray(profiles, np.float32).reshape(-1, nbins)
    w = np.ascontiguousarray(widths, np.uint64)
    return np.array([lib().lko_snr_max_div(_p(np.ascontiguousarray(r)), nbins, _p(w), w.size, stdnoise)
                     for r in p], np.float32)


def mc_stage(folds_in, noise, signal, var_in, var_add, widths, threshold, thresholds=(), src=None,
             signal_scale=1.0, rowmap=None, ntrials=None, cls=None):
    """simulate_score_prune_fused: returns (survivor folds, survivor noise rows,
    counts per threshold of the grid (then of the flagged rows, with cls),
    max S/N per trial)."""
    fin = np.ascontiguousarray(folds_in, np.float32)
    nz = np.ascontiguousarray(noise, np.float32)
    nbins = nz.shape[-1]
    rm = None if rowmap is None else np.ascontiguousarray(rowmap, np.uint32)
    if ntrials is None:
        ntrials = rm.size if rm is not None else nz.shape[0]
    sg = np.ascontiguousarray(signal, np.float32)
    per_trial = int(sg.ndim == 2)
    w = np.ascontiguousarray(widths, np.uint64)
    thr = np.ascontiguousarray(thresholds, np.float32)
    s = None if src is None else np.ascontiguousarray(src, np.uint32)
    out = np.zeros((ntrials, nbins), np.float32)
    ids = np.zeros(ntrials, np.uint32)
    c = None if cls is None else np.ascontiguousarray(cls, np.uint8)
    ncnt = thr.size * (2 if c is not None else 1)
    counts = np.zeros(max(ncnt, 1), np.uint64)
    mx = np.zeros(ntrials, np.float32)
    k = lib().lko_mc_stage(_p(fin), None if s is None else _p(s), ntrials, nbins, _p(nz), _p(sg), per_trial,
                           signal_scale, None if rm is None else _p(rm), var_in, var_add, _p(w), w.size,
                           threshold, _p(thr), thr.size, None if c is None else _p(c), _p(out), _p(ids),
                           _p(counts), _p(mx))
    return out[:k], ids[:k], counts[:ncnt], mx


# ---- DynamicThresholdScheme beam search -------------------------------------

DTS_STATE_DTYPE = np.dtype([("success_h0", np.float32), ("success_h1", np.float32), ("complexity", np.float32),
                            ("complexity_cumul", np.float32), ("success_h1_cumul", np.float32),
                            ("nbranches", np.float32), ("threshold", np.float32), ("cost", np.float32),
                            ("threshold_prev", np.float32), ("success_h1_cumul_prev", np.float32),
                            ("is_empty", np.bool_), ("_pad", np.uint8, 3)])
DTS_LUT_SIZE = (1 << 17) + 1


class DtsCfg(ctypes.Structure):
    _fields_ = [("branching_pattern", vp), ("nstages", u32), ("ref_ducy", f32), ("nbins", u32), ("ntrials", u32),
                ("nprobs", u32), ("prob_min", f32), ("snr_final", f32), ("nthresholds", u32), ("ducy_max", f32),
                ("wtsp", f32), ("beam_width", f32), ("trials_start", u32), ("seed", u64)]


def _dts_lib():
    L = lib()
    if not hasattr(L, "_dts_ready"):
        L.lko_normal_quantile.restype = f64
        L.lko_normal_quantile.argtypes = [f64]
        L.lko_dts_normal_lut.argtypes = [vp]
        L.lko_dts_thresholds.argtypes = [f32, f32, u32, vp]
        L.lko_dts_probs.argtypes = [u32, f32, vp]
        L.lko_dts_profile.argtypes = [u32, f32, f32, vp]
        L.lko_dts_guess.argtypes = [u32, f32, vp, u32, f32, vp]
        L.lko_dts_neighbours.restype = u32
        L.lko_dts_neighbours.argtypes = [vp, u32, u32, u32, vp]
        L.lko_dts_lower_bin.restype = ctypes.c_int64
        L.lko_dts_lower_bin.argtypes = [vp, u32, f32]
        L.lko_philox4x32_10.argtypes = [vp, u32, u32, vp]
        L.lko_dts_normal.restype = f32
        L.lko_dts_normal.argtypes = [u32, vp]
        L.lko_dts_resample.restype = u32
        L.lko_dts_resample.argtypes = [u32, u32, u32, u32, u32, u32]
        L.lko_dts_run.argtypes = [vp, u32, u32, vp]
        L._dts_ready = True
    return L


def dts_normal_lut() -> np.ndarray:
    out = np.zeros(DTS_LUT_SIZE, np.float32)
    _dts_lib().lko_dts_normal_lut(_p(out))
    return out


def dts_thresholds(snr_start, snr_final, n) -> np.ndarray:
    out = np.zeros(n, np.float32)
    _dts_lib().lko_dts_thresholds(snr_start, snr_final, n, _p(out))
    return out


def dts_probs(n, prob_min) -> np.ndarray:
    out = np.zeros(n, np.float32)
    _dts_lib().lko_dts_probs(n, prob_min, _p(out))
    return out


def dts_profile(nbins, ducy, center=0.5) -> np.ndarray:
    out = np.zeros(nbins, np.float32)
    _dts_lib().lko_dts_profile(nbins, ducy, center, _p(out))
    return out


def dts_guess(nstages, snr_bound, branching, trials_start=1, min_trials=1e10) -> np.ndarray:
    b = np.ascontiguousarray(branching, np.float32)
    out = np.zeros(nstages, np.float32)
    _dts_lib().lko_dts_guess(nstages, snr_bound, _p(b), trials_start, min_trials, _p(out))
    return out


def dts_neighbours(indices, target, num) -> np.ndarray:
    idx = np.ascontiguousarray(indices, np.uint32)
    out = np.zeros(num + 1, np.uint32)
    n = _dts_lib().lko_dts_neighbours(_p(idx), idx.size, target, num, _p(out))
    return out[:n].copy()


def dts_lower_bin(range_, value) -> int:
    r = np.ascontiguousarray(range_, np.float32)
    return int(_dts_lib().lko_dts_lower_bin(_p(r), r.size, value))


def philox4x32_10(ctr, seed) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    _dts_lib().lko_philox4x32_10(_p(c), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, _p(out))
    return out


def dts_run(branching, ref_ducy, nbins=64, ntrials=1024, nprobs=10, prob_min=0.05, snr_final=8.0, nthresholds=100,
            ducy_max=0.3, wtsp=1.0, beam_width=0.7, trials_start=1, seed=0x10C1B200, thres_neigh=10,
            stages_run=0) -> np.ndarray:
    """The beam search (its first stages_run stages; 0: all); states
    [nstages * nthresholds * nprobs]."""
    b = np.ascontiguousarray(branching, np.float32)
    cfg = DtsCfg(_p(b), b.size, ref_ducy, nbins, ntrials, nprobs, prob_min, snr_final, nthresholds, ducy_max, wtsp,
                 beam_width, trials_start, seed)
    out = np.zeros(b.size * nthresholds * nprobs, DTS_STATE_DTYPE)
    _check(_dts_lib().lko_dts_run(ctypes.byref(cfg), thres_neigh, stages_run, _p(out)))
    return out
