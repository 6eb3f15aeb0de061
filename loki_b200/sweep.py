"""Frequency sweep over octave regions: ``generate_ffa_regions``,
``FFARegionPlannerTime`` and ``FFAFreqSweepCUDA``, mirroring the reference's
``libloki.plans.generate_ffa_regions`` / ``FFARegionPlannerTime``
(src/loki_python.cpp:481-520, lib/regions.cpp) and
``libculoki.ffa.FFAFreqSweepCUDA`` (src/loki_python_cuda.cpp:205-218,
lib/ffa_freq_sweep_cuda.cu).

The planner cuts ``[f_min, f_max]`` into octave regions (nbins growing with
the period, constant duty-cycle resolution) and each region into chunks that
fit ``cfg.max_process_memory_gb`` under the reference's memory model; the
sweep runs FFA + boxcar scores + ``>= snr_min`` compaction per chunk on the
GPU and decodes every passing (coordinate, width) into parameter values.
The reference writes the candidates to ``{prefix}_ffa_results.h5``; here
``execute`` writes the same datasets (``param_sets``, ``snr``) and
attributes (``param_names``, ``scoring_widths``) to
``{prefix}_ffa_results.npz`` and also returns them.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _capi as C
from . import _device as D
from .configs import PulsarSearchConfig

_STORAGE = {"fp32": C.LK_FP32, "float32": C.LK_FP32, "bf16": C.LK_BF16, "fp16": C.LK_FP16}


FFA_REGION_DTYPE = np.dtype([("f_start", np.float64), ("f_end", np.float64), ("nbins", np.uint64),
                             ("eta", np.float64)])


def generate_ffa_regions(p_min: float, p_max: float, tsamp: float, nbins_min: int, eta_min: float,
                         growth_factor: float = 2.0, nbins_max: int | None = None) -> np.ndarray:
    """Octave regions (lib/regions.cpp:31-78) as a structured array of
    (f_start, f_end, nbins, eta)."""
    nmax = 1024 if nbins_max is None else int(nbins_max)
    n = ctypes.c_uint64()
    C.check(C.lib().lk_generate_ffa_regions(p_min, p_max, tsamp, int(nbins_min), eta_min, growth_factor, nmax,
                                            None, 0, ctypes.byref(n)))
    rows = np.zeros((n.value, 4), np.float64)
    C.check(C.lib().lk_generate_ffa_regions(p_min, p_max, tsamp, int(nbins_min), eta_min, growth_factor, nmax,
                                            rows.ctypes.data, n.value, ctypes.byref(n)))
    out = np.zeros(n.value, FFA_REGION_DTYPE)
    out["f_start"], out["f_end"], out["nbins"], out["eta"] = rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 3]
    return out


_EXECUTORS = {None: 0, "auto": 0, "resident": 1, "one_at_a_time": 2}


def _options(cfg: PulsarSearchConfig, device_model: bool, decode_chunk_widths: bool,
             executors=None, autotune: bool = False, plan_sizes: int = 0) -> C.LkSweepOptions:
    o = C.LkSweepOptions()
    o.max_memory_gb = cfg.max_process_memory_gb
    o.octave_scale = cfg.octave_scale
    o.nbins_max = cfg.nbins_max
    o.max_passing_candidates = cfg.max_passing_candidates
    o.decode_chunk_widths = int(bool(decode_chunk_widths))
    o.device_memory_model = int(bool(device_model))
    if executors not in _EXECUTORS:
        raise ValueError(f"executors must be one of {sorted(k for k in _EXECUTORS if k)}")
    o.executor_mode = _EXECUTORS[executors]
    o.autotune = int(bool(autotune))
    o.use_fourier = int(bool(cfg.use_fourier))
    o.nbins_min_lossy_bf = int(cfg.nbins_min_lossy_bf)
    o.plan_sizes = int(plan_sizes)
    return o


class _SweepHandle:
    def __init__(self, cfg: PulsarSearchConfig, device_id: int, storage: int, device_model: bool,
                 decode_chunk_widths: bool, executors=None, autotune: bool = False, plan_sizes: int = 0):
        self._cfg = cfg
        self._opt = _options(cfg, device_model, decode_chunk_widths, executors, autotune, plan_sizes)
        h = ctypes.c_void_p()
        C.check(C.lib().lk_sweep_create(ctypes.byref(cfg.c_config), ctypes.byref(self._opt), device_id, storage,
                                        ctypes.byref(h)))
        self._h = h
        n = ctypes.c_uint64()
        C.check(C.lib().lk_sweep_nchunks(h, ctypes.byref(n)))
        self._chunks = []
        for i in range(n.value):
            ch = C.LkSweepChunk()
            C.check(C.lib().lk_sweep_chunk_info(h, i, ctypes.byref(ch)))
            self._chunks.append({k: getattr(ch, k) for k, _ in C.LkSweepChunk._fields_})

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                C.lib().lk_sweep_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def nregions(self) -> int:
        return len(self._chunks)

    @property
    def chunks(self) -> list[dict]:
        """Per chunk: drift-widened (f_min, f_max), nominal range, nbins, eta,
        plan sizes and memory (GB)."""
        return [dict(c) for c in self._chunks]

    @property
    def cfgs(self) -> list[PulsarSearchConfig]:
        """The chunk configurations (reference ``get_cfgs``)."""
        out = []
        for c in self._chunks:
            lim = np.array(self._cfg.param_limits, dtype=np.float64)
            lim[-1] = (c["f_min"], c["f_max"])
            out.append(self._cfg.get_updated_config(int(c["nbins"]), float(c["eta"]), lim))
        return out

    @property
    def max_sizes(self) -> dict:
        """The workspace sizes of the largest chunk (reference ``FFARegionStats``)."""
        if not self._chunks:
            return {"max_buffer_size": 0, "max_coord_size": 0, "max_ncoords": 0, "max_ffa_levels": 0,
                    "freq_sweep_memory_usage": 0.0}
        return {
            "max_buffer_size": max(c["buffer_size"] for c in self._chunks),
            "max_coord_size": max(c["coord_size"] for c in self._chunks),
            "max_ncoords": max(c["ncoords"] for c in self._chunks),
            "max_ffa_levels": max(c["n_levels"] for c in self._chunks),
            "freq_sweep_memory_usage": self._chunks[-1]["allocated_gb"],
        }


class FFARegionPlannerTime(_SweepHandle):
    """Chunk plan of a frequency sweep (reference ``FFARegionPlannerTime``,
    FFARegionPlanner<float>: fold buffers sized in nbins per row; a
    ``use_fourier`` configuration counts them 8 bytes each, as there).
    ``use_gpu`` selects the device memory model of FFAFreqSweepCUDA (else the
    process model of FFAFreqSweep). Planning touches no device."""

    def __init__(self, cfg: PulsarSearchConfig, use_gpu: bool = False):
        super().__init__(cfg, 0, C.LK_FP32, use_gpu, False, plan_sizes=1)

    def get_cfgs(self) -> list[PulsarSearchConfig]:
        return self.cfgs

    def get_nregions(self) -> int:
        return self.nregions


class FFARegionPlannerFourier(FFARegionPlannerTime):
    """Chunk plan of the Fourier-domain sweep (reference
    ``FFARegionPlannerFourier``, FFARegionPlanner<ComplexType>: fold buffers
    sized in nbins // 2 + 1 complex harmonics per row)."""

    def __init__(self, cfg: PulsarSearchConfig, use_gpu: bool = False):
        _SweepHandle.__init__(self, cfg, 0, C.LK_FP32, use_gpu, False, plan_sizes=2)


class FFAFreqSweepCUDA(_SweepHandle):
    """Frequency sweep on one device (reference ``FFAFreqSweepCUDA``).

    Extensions: ``fold_storage`` ("fp32" or "bf16": intermediate fold levels
    in BF16, candidates identical to FP32), ``decode_chunk_widths`` (decode
    each chunk's candidates with that chunk's own width list instead of the
    base configuration's, which is what the reference does) and
    ``device_memory_model`` (False: chunk with FFAFreqSweep's process model) and
    ``executors`` (None / "auto": every chunk's executor kept on the device when
    they all fit in free memory with room to spare, else one chunk at a time;
    "resident"; "one_at_a_time": at most one chunk's workspace on the device,
    the planner's budget) and ``autotune`` (each chunk executor's launch
    shapes timed on the first run's series and kept). The results depend on
    neither.
    """

    def __init__(self, cfg: PulsarSearchConfig, device_id: int = 0, fold_storage: str = "fp32",
                 decode_chunk_widths: bool = False, device_memory_model: bool = True, executors=None,
                 autotune: bool = False):
        D.require_cuda(device_id)
        if fold_storage not in _STORAGE:
            raise ValueError(f"fold_storage must be one of {sorted(_STORAGE)}")
        self._device = device_id
        with D.torch().cuda.device(device_id):
            super().__init__(cfg, device_id, _STORAGE[fold_storage], device_memory_model, decode_chunk_widths,
                             executors, autotune)
        self._param_sets = np.zeros((0, cfg.nparams + 1))
        self._snr = np.zeros(0, np.float32)
        self._region_counts = np.zeros(self.nregions, np.uint64)

    def run(self, ts_e, ts_v) -> tuple[np.ndarray, np.ndarray]:
        """Search every chunk; returns (param_sets [n, nparams + 1], snr [n])."""
        n = self._cfg.nsamps
        e = D.to_device_f32(ts_e, self._device)
        v = D.to_device_f32(ts_v, self._device)
        if e.numel() != n or v.numel() != n:
            raise RuntimeError("FFAFreqSweep::execute: ts_e and ts_v must have size nsamps")
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_sweep_execute(self._h, D.ptr(e), D.ptr(v), D.stream_ptr(self._device)))
        total = ctypes.c_uint64()
        C.check(C.lib().lk_sweep_results(self._h, None, None, 0, ctypes.byref(total), None))
        k = total.value
        stride = self._cfg.nparams + 1
        params = np.zeros(k * stride, np.float64)
        snr = np.zeros(k, np.float32)
        counts = np.zeros(self.nregions, np.uint64)
        C.check(C.lib().lk_sweep_results(self._h, params.ctypes.data, snr.ctypes.data, k, ctypes.byref(total),
                                         counts.ctypes.data))
        self._param_sets = params.reshape(k, stride)
        self._snr = snr
        self._region_counts = counts
        return self._param_sets, self._snr

    def set_profiling(self, enable: bool = True) -> None:
        """Record CUDA events around every kernel stage of every chunk."""
        C.check(C.lib().lk_sweep_set_profiling(self._h, 1 if enable else 0))

    def profile(self) -> list[dict]:
        """Stages of the last run summed by kind over levels and chunks."""
        arr = (C.LkStageTime * 16)()
        n = ctypes.c_uint32()
        C.check(C.lib().lk_sweep_get_profile(self._h, arr, 16, ctypes.byref(n)))
        return [{"stage": C.STAGE_NAMES.get(arr[i].kind, str(arr[i].kind)), "launches": arr[i].launches,
                 "ms": float(arr[i].ms), "bytes": int(arr[i].bytes)} for i in range(min(n.value, 16))]

    @property
    def region_counts(self) -> np.ndarray:
        """Passing candidates per chunk of the last run."""
        return self._region_counts.copy()

    def execute(self, ts_e, ts_v, outdir: str = "./", file_prefix: str = "test") -> str:
        """Run and write ``{outdir}/{file_prefix}_ffa_results.npz`` (the
        reference's HDF5 datasets and attributes); returns the path."""
        params, snr = self.run(ts_e, ts_v)
        names = list(self._cfg.param_names) + ["width"]
        path = os.path.join(outdir, f"{file_prefix}_ffa_results.npz")
        np.savez(path, param_sets=params, snr=snr, param_names=np.array(names),
                 scoring_widths=np.asarray(self._cfg.score_widths, np.uint64),
                 region_counts=self._region_counts,
                 chunk_f_limits=np.array([[c["f_min"], c["f_max"]] for c in self._chunks]).reshape(-1, 2),
                 chunk_nbins=np.array([c["nbins"] for c in self._chunks], np.uint64))
        return path
