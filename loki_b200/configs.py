"""``PulsarSearchConfig``: the search configuration, mirroring
``libloki.configs.PulsarSearchConfig`` of the reference (bound at
src/loki_python.cpp:277-373, implemented in lib/configs.cpp).

Validation and every derived quantity (bseg_brute default, level count, grid
steps, width trials) come from the native plan code, so a configuration the
reference rejects raises here too, with the reference's message.
"""

from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _capi as C

# include/loki/common/types.hpp kParamNames, last nparams entries are used.
_PARAM_NAMES = ("crackle", "snap", "jerk", "accel", "freq")


class PulsarSearchConfig:
    """Search configuration (same constructor arguments as the reference).

    Extensions: ``score_widths`` (explicit boxcar widths instead of
    ``generate_box_width_trials(nbins, ducy_max, wtsp)``).
    """

    def __init__(
        self,
        nsamps: int,
        tsamp: float,
        nbins: int,
        eta: float,
        param_limits,
        ducy_max: float = 0.2,
        wtsp: float = 1.5,
        use_fourier: bool = True,
        nthreads: int = 1,
        max_process_memory_gb: float = 8.0,
        octave_scale: float = 2.0,
        nbins_max: int = 1024,
        nbins_min_lossy_bf: int = 64,
        bseg_brute: int | None = None,
        bseg_ffa: int | None = None,
        snr_min: float = 5.0,
        max_passing_candidates: int = 1 << 22,
        prune_poly_order: int = 3,
        p_orb_min: float = 1e-5,
        m_c_max: float = 10.0,
        m_p_min: float = 1.4,
        minimum_snap_cells: float = 5.0,
        use_conservative_tile: bool = False,
        score_widths: Sequence[int] | None = None,
    ):
        lim = np.asarray(param_limits, dtype=np.float64)
        if lim.ndim != 2 or lim.shape[1] != 2:
            raise ValueError("param_limits must be a 2D NumPy array with shape (n_params, 2)")
        if lim.shape[0] == 0:
            raise RuntimeError("coord_limits must be non-empty")
        if nbins_max < nbins:
            raise RuntimeError("nbins_max must be greater than or equal to nbins")
        if max_process_memory_gb <= 0:
            raise RuntimeError("max_process_memory_gb must be positive")
        self._nsamps = int(nsamps)
        self._tsamp = float(tsamp)
        self._nbins = int(nbins)
        self._eta = float(eta)
        self._param_limits = lim.copy()
        self._ducy_max = float(ducy_max)
        self._wtsp = float(wtsp)
        self._use_fourier = bool(use_fourier)
        self._nthreads = max(1, int(nthreads))
        self._max_process_memory_gb = float(max_process_memory_gb)
        self._octave_scale = float(octave_scale)
        self._nbins_max = int(nbins_max)
        self._nbins_min_lossy_bf = int(nbins_min_lossy_bf)
        self._snr_min = float(snr_min)
        self._max_passing_candidates = int(max_passing_candidates)
        self._prune_poly_order = int(prune_poly_order)
        self._p_orb_min = float(p_orb_min)
        self._m_c_max = float(m_c_max)
        self._m_p_min = float(m_p_min)
        self._minimum_snap_cells = float(minimum_snap_cells)
        self._use_conservative_tile = bool(use_conservative_tile)
        self._bseg_brute_explicit = bseg_brute
        self._bseg_ffa_explicit = bseg_ffa
        self._score_widths_explicit = None if score_widths is None else [int(w) for w in score_widths]

        c = C.LkConfig()
        c.nsamps = self._nsamps
        c.tsamp = self._tsamp
        c.nbins = self._nbins
        c.eta = self._eta
        c.nparams = lim.shape[0]
        if lim.shape[0] > C.LK_MAX_PARAMS:
            raise RuntimeError(f"nparams must be <= {C.LK_MAX_PARAMS}")
        for i, (a, b) in enumerate(lim):
            c.param_limits[2 * i] = a
            c.param_limits[2 * i + 1] = b
        c.ducy_max = self._ducy_max
        c.wtsp = self._wtsp
        c.bseg_brute = int(bseg_brute) if bseg_brute else 0
        c.bseg_ffa = int(bseg_ffa) if bseg_ffa else 0
        c.snr_min = self._snr_min
        if self._score_widths_explicit is not None:
            w = self._score_widths_explicit
            if not 1 <= len(w) <= C.LK_MAX_WIDTHS:
                raise RuntimeError(f"score_widths must hold 1..{C.LK_MAX_WIDTHS} widths")
            c.n_score_widths = len(w)
            for i, x in enumerate(w):
                c.score_widths[i] = x
        self._c = c
        h = ctypes.c_void_p()
        C.check(C.lib().lk_plan_create(ctypes.byref(c), ctypes.byref(h)))
        self._plan_handle = h
        info = C.LkPlanInfo()
        C.check(C.lib().lk_plan_get_info(h, ctypes.byref(info)))
        self._info = info

    def __del__(self):
        h = getattr(self, "_plan_handle", None)
        if h is not None and h.value:
            try:
                C.lib().lk_plan_destroy(h)
            except Exception:
                pass
            self._plan_handle = None

    # -- the raw C struct, for the plan / executor classes ------------------
    @property
    def c_config(self) -> C.LkConfig:
        return self._c

    # -- properties of the reference ---------------------------------------
    nsamps = property(lambda self: self._nsamps)
    tsamp = property(lambda self: self._tsamp)
    nbins = property(lambda self: self._nbins)
    eta = property(lambda self: self._eta)
    ducy_max = property(lambda self: self._ducy_max)
    wtsp = property(lambda self: self._wtsp)
    use_fourier = property(lambda self: self._use_fourier)
    nthreads = property(lambda self: self._nthreads)
    max_process_memory_gb = property(lambda self: self._max_process_memory_gb)
    octave_scale = property(lambda self: self._octave_scale)
    nbins_max = property(lambda self: self._nbins_max)
    nbins_min_lossy_bf = property(lambda self: self._nbins_min_lossy_bf)
    snr_min = property(lambda self: self._snr_min)
    max_passing_candidates = property(lambda self: self._max_passing_candidates)
    prune_poly_order = property(lambda self: self._prune_poly_order)
    p_orb_min = property(lambda self: self._p_orb_min)
    m_c_max = property(lambda self: self._m_c_max)
    m_p_min = property(lambda self: self._m_p_min)
    minimum_snap_cells = property(lambda self: self._minimum_snap_cells)
    use_conservative_tile = property(lambda self: self._use_conservative_tile)

    @property
    def tobs(self) -> float:
        return float(self._nsamps) * self._tsamp

    @property
    def nbins_f(self) -> int:
        return self._nbins // 2 + 1

    @property
    def param_limits(self) -> np.ndarray:
        return self._param_limits.copy()

    @property
    def nparams(self) -> int:
        return int(self._info.nparams)

    @property
    def param_names(self) -> list[str]:
        return list(_PARAM_NAMES[len(_PARAM_NAMES) - self.nparams :])

    @property
    def f_min(self) -> float:
        return float(self._param_limits[-1, 0])

    @property
    def f_max(self) -> float:
        return float(self._param_limits[-1, 1])

    @property
    def bseg_brute(self) -> int:
        return int(self._info.bseg_brute)

    @property
    def bseg_ffa(self) -> int:
        return int(self._info.bseg_ffa)

    @property
    def tseg_brute(self) -> float:
        return float(self._info.tseg_brute)

    @property
    def tseg_ffa(self) -> float:
        return float(self._info.tseg_ffa)

    @property
    def niters_ffa(self) -> int:
        return int(self._info.n_levels) - 1

    @property
    def score_widths(self) -> np.ndarray:
        return np.array(self._info.widths[: self._info.n_widths], dtype=np.uint64)

    @property
    def n_scoring_widths(self) -> int:
        return int(self._info.n_widths)

    def _dparams(self, tseg_cur: float, kind: int) -> np.ndarray:
        out = np.zeros(self.nparams, dtype=np.float64)
        C.check(C.lib().lk_plan_dparams(self._plan_handle, float(tseg_cur), kind, out.ctypes.data))
        return out

    def dparams(self, tseg_cur: float) -> np.ndarray:
        return self._dparams(tseg_cur, 0)

    def dparams_f(self, tseg_cur: float) -> np.ndarray:
        return self._dparams(tseg_cur, 1)

    def dparams_actual(self, tseg_cur: float) -> np.ndarray:
        return self._dparams(tseg_cur, 2)

    def get_updated_config(self, nbins: int, eta: float, param_limits) -> "PulsarSearchConfig":
        """Same configuration with new nbins / eta / param_limits (lib/configs.cpp:186-223)."""
        return PulsarSearchConfig(
            self._nsamps, self._tsamp, nbins, eta, param_limits, self._ducy_max, self._wtsp,
            self._use_fourier, self._nthreads, self._max_process_memory_gb, self._octave_scale,
            self._nbins_max, self._nbins_min_lossy_bf, self._bseg_brute_explicit,
            self._bseg_ffa_explicit, self._snr_min, self._max_passing_candidates,
            self._prune_poly_order, self._p_orb_min, self._m_c_max, self._m_p_min,
            self._minimum_snap_cells, self._use_conservative_tile, self._score_widths_explicit,
        )

    def __repr__(self) -> str:
        return (
            f"PulsarSearchConfig(nsamps={self._nsamps}, tsamp={self._tsamp}, nbins={self._nbins}, "
            f"eta={self._eta}, param_limits={self._param_limits.tolist()}, "
            f"bseg_brute={self.bseg_brute}, levels={self.niters_ffa + 1})"
        )
