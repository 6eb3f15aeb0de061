"""Monte-Carlo threshold stages on the GPU (the inner step of the reference's
``DynamicThresholdScheme``: ``simulate_score_prune_fused``,
lib/thresholds.cpp:358-431, with ``snr_boxcar_threshold_with_cache``,
lib/score.cpp:434-462).

One stage turns every trial's fold into the next stage's fold
``(in + noise) + signal * scale``, scores it (largest boxcar S/N over the
widths, each divided by ``sqrt(var_in + var_add)``), counts it against a grid
of up to 64 thresholds and keeps the trials above the pruning threshold in
trial order. The noise is an input, drawn on the host, so the CPU reference
can be run on the same numbers (the reference seeds its own generator from
``std::random_device``).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from . import _device as D


class MCStageCUDA:
    """Fused Monte-Carlo stage executor for up to ``max_trials`` trials of ``nbins`` bins."""

    def __init__(self, max_trials: int, nbins: int, widths, device_id: int = 0):
        D.require_cuda(device_id)
        self._w = np.ascontiguousarray(widths, dtype=np.uint32)
        self._nbins = int(nbins)
        self._device = device_id
        self._max = int(max_trials)
        h = ctypes.c_void_p()
        with D.torch().cuda.device(device_id):
            C.check(C.lib().lk_mc_create(self._max, self._nbins, self._w.ctypes.data, self._w.size, device_id,
                                         ctypes.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                C.lib().lk_mc_destroy(h)
            except Exception:
                pass
            self._h = None

    def status(self) -> int:
        """Synchronises; non-zero when a src / rowmap index was out of range
        since the last call (the flag is cleared)."""
        st = ctypes.c_uint32()
        C.check(C.lib().lk_mc_status(self._h, D.stream_ptr(self._device), ctypes.byref(st)))
        return st.value

    def stage(self, folds_in, noise, signal, threshold: float, var_in: float, var_add: float,
              thresholds=(), signal_scale: float = 1.0, rowmap=None, src=None, ntrials: int | None = None,
              cls=None, folds_out=None, with_max_snr: bool = False):
        """Runs one stage on CUDA tensors (host arrays are copied in). Returns a
        dict of device tensors: ``folds`` (survivors first), ``ids`` (noise row of
        each survivor), ``count`` (int64[1]), ``counts`` (uint64 grid counts as
        int64, twice as long with ``cls``), ``max_snr`` (with ``with_max_snr``)."""
        t = D.torch()
        dev = f"cuda:{self._device}"

        def u32(x):
            if x is None:
                return None
            if isinstance(x, t.Tensor):
                return x.to(device=dev, dtype=t.int32).contiguous()
            return t.from_numpy(np.ascontiguousarray(x, dtype=np.uint32).view(np.int32)).to(dev)

        fin = D.to_device_f32(folds_in, self._device)
        nz = D.to_device_f32(noise, self._device)
        sg = D.to_device_f32(signal, self._device)
        rm = u32(rowmap)
        sr = u32(src)
        if ntrials is None:
            ntrials = rm.numel() if rm is not None else nz.numel() // self._nbins
        per_trial = 1 if sg.numel() > self._nbins else 0
        thr = np.ascontiguousarray(thresholds, dtype=np.float32)
        cl = None
        if cls is not None:
            cl = cls.to(device=dev, dtype=t.uint8).contiguous() if isinstance(cls, t.Tensor) else \
                t.from_numpy(np.ascontiguousarray(cls, dtype=np.uint8)).to(dev)
        out = folds_out if folds_out is not None else t.empty((max(ntrials, 1), self._nbins), dtype=t.float32,
                                                               device=dev)
        ids = t.empty(max(ntrials, 1), dtype=t.int32, device=dev)
        count = t.zeros(1, dtype=t.int64, device=dev)
        counts = t.zeros(max(thr.size * (2 if cl is not None else 1), 1), dtype=t.int64, device=dev)
        mx = t.empty(max(ntrials, 1), dtype=t.float32, device=dev) if with_max_snr else None
        with t.cuda.device(self._device):
            C.check(C.lib().lk_mc_stage(
                self._h, D.ptr(fin), fin.numel() // self._nbins, None if sr is None else sr.data_ptr(),
                int(ntrials), D.ptr(nz), nz.numel() // self._nbins, D.ptr(sg), per_trial, float(signal_scale),
                None if rm is None else rm.data_ptr(), float(var_in), float(var_add), float(threshold), thr.ctypes.data if thr.size else None, thr.size,
                None if cl is None else cl.data_ptr(), out.data_ptr(), ids.data_ptr(), count.data_ptr(),
                counts.data_ptr(), None if mx is None else mx.data_ptr(), D.stream_ptr(self._device)))
        res = {"folds": out, "ids": ids, "count": count, "counts": counts[: thr.size * (2 if cl is not None else 1)]}
        if mx is not None:
            res["max_snr"] = mx[:ntrials]
        return res


def simulate_score_prune_fused(folds_in, profile, noise, threshold: float, widths, var_in: float,
                               bias_snr: float = 0.0, var_add: float = 1.0, device_id: int = 0):
    """The reference's fused step for one shared signal shape (``profile *
    bias_snr``) and ntrials == ntrials_in: returns (survivor folds as a host
    array, success fraction)."""
    nz = np.ascontiguousarray(noise, dtype=np.float32)
    ntrials, nbins = nz.shape
    sig = (np.ascontiguousarray(profile, dtype=np.float32) * np.float32(bias_snr)).astype(np.float32)
    st = MCStageCUDA(ntrials, nbins, widths, device_id)
    r = st.stage(folds_in, nz, sig, threshold, var_in, var_add)
    k = int(r["count"].item())
    return r["folds"][:k].cpu().numpy(), k / ntrials


def mc_cascade(folds0, signal, noises, cls, widths, thresholds, grids, var0: float = 1.0,
               device_id: int = 0):
    """Runs a cascade of stages: stage s adds noises[s] (variance doubling, so
    var_add = var of the input) and the signal times 2**s, keeps the trials
    whose S/N exceeds thresholds[s] and counts all / flagged trials against
    grids[s]. Inputs may be host arrays or CUDA tensors (noises: one
    [ntrials0, nbins] array per stage, indexed by the original trial).
    Returns a list of per-stage dicts (alive, kept, counts, counts_flagged)."""
    t = D.torch()
    dev = f"cuda:{device_id}"
    f0 = D.to_device_f32(folds0, device_id)
    n0, nbins = f0.shape
    st = MCStageCUDA(n0, nbins, widths, device_id)
    sig = D.to_device_f32(signal, device_id)
    cl = cls if isinstance(cls, t.Tensor) else t.from_numpy(np.ascontiguousarray(cls, dtype=np.uint8)).to(dev)
    rows = t.arange(n0, dtype=t.int32, device=dev)
    buf = [f0, t.empty_like(f0)]
    cur, alive, var = 0, n0, float(var0)
    out = []
    for s, nz in enumerate(noises):
        r = st.stage(buf[cur], nz, sig, float(thresholds[s]), var, var, thresholds=grids[s],
                     signal_scale=float(2 ** s), rowmap=rows[:alive], ntrials=alive, cls=cl,
                     folds_out=buf[1 - cur])
        kept = int(r["count"].item())
        if st.status() != 0:
            raise RuntimeError("mc_cascade: a trial row index was out of range")
        g = len(grids[s])
        counts = r["counts"].cpu().numpy()
        out.append({"stage": s, "alive": alive, "kept": kept, "var": 2 * var,
                    "counts": counts[:g], "counts_flagged": counts[g:]})
        rows = r["ids"][:kept].clone()
        cur, alive, var = 1 - cur, kept, 2 * var
        if alive == 0:
            break
    return out


# detection::State (include/loki/detection/thresholds.hpp:17-29); the
# reference's pybind module exposes get_states() with these fields.
STATE_DTYPE = np.dtype([("success_h0", np.float32), ("success_h1", np.float32), ("complexity", np.float32),
                        ("complexity_cumul", np.float32), ("success_h1_cumul", np.float32),
                        ("nbranches", np.float32), ("threshold", np.float32), ("cost", np.float32),
                        ("threshold_prev", np.float32), ("success_h1_cumul_prev", np.float32),
                        ("is_empty", np.bool_), ("_pad", np.uint8, 3)])


class _DtsConfig(ctypes.Structure):
    _fields_ = [("branching_pattern", ctypes.c_void_p), ("nstages", ctypes.c_uint32), ("ref_ducy", ctypes.c_float),
                ("nbins", ctypes.c_uint32), ("ntrials", ctypes.c_uint32), ("nprobs", ctypes.c_uint32),
                ("prob_min", ctypes.c_float), ("snr_final", ctypes.c_float), ("nthresholds", ctypes.c_uint32),
                ("ducy_max", ctypes.c_float), ("wtsp", ctypes.c_float), ("beam_width", ctypes.c_float),
                ("trials_start", ctypes.c_uint32), ("seed", ctypes.c_uint64)]


DEFAULT_SEED = 0x10C1B200


class DynamicThresholdSchemeCUDA:
    """The reference's ``DynamicThresholdSchemeCUDA`` / ``DynamicThresholdScheme``
    (lib/thresholds.cpp:560-907): beam search over (stage x threshold x
    probability bin) with simulated H0 / H1 folds. Same arguments
    (``batch_size`` is accepted and unused: every transition of a stage runs
    in one launch); ``seed`` fixes the counter-based noise, so a run is
    reproducible and matches the CPU oracle's."""

    def __init__(self, branching_pattern, ref_ducy: float, nbins: int = 64, ntrials: int = 1024, nprobs: int = 10,
                 prob_min: float = 0.05, snr_final: float = 8.0, nthresholds: int = 100, ducy_max: float = 0.3,
                 wtsp: float = 1.0, beam_width: float = 0.7, trials_start: int = 1, batch_size: int = 256,
                 device_id: int = 0, seed: int = DEFAULT_SEED):
        D.require_cuda(device_id)
        self._bp = np.ascontiguousarray(branching_pattern, dtype=np.float32)
        if self._bp.size == 0:
            raise ValueError("Branching pattern is empty")
        cfg = _DtsConfig(self._bp.ctypes.data, self._bp.size, float(ref_ducy), int(nbins), int(ntrials), int(nprobs),
                         float(prob_min), float(snr_final), int(nthresholds), float(ducy_max), float(wtsp),
                         float(beam_width), int(trials_start), int(seed))
        self._device = device_id
        h = ctypes.c_void_p()
        with D.torch().cuda.device(device_id):
            C.check(C.lib().lk_dts_create(ctypes.byref(cfg), device_id, ctypes.byref(h)))
        self._h = h
        ns, nt, npb, nb, nw = (ctypes.c_uint32() for _ in range(5))
        C.check(C.lib().lk_dts_info(h, ctypes.byref(ns), ctypes.byref(nt), ctypes.byref(npb), ctypes.byref(nb),
                                    ctypes.byref(nw)))
        self.nstages, self.nthresholds, self.nprobs = ns.value, nt.value, npb.value
        self._nbins, self._nw = nb.value, nw.value
        self.profile = np.zeros(self._nbins, np.float32)
        self.thresholds = np.zeros(self.nthresholds, np.float32)
        self.probs = np.zeros(self.nprobs, np.float32)
        self.guess_path = np.zeros(self.nstages, np.float32)
        self.box_score_widths = np.zeros(self._nw, np.uint32)
        C.check(C.lib().lk_dts_arrays(h, self.profile.ctypes.data, self.thresholds.ctypes.data,
                                      self.probs.ctypes.data, self.guess_path.ctypes.data,
                                      self.box_score_widths.ctypes.data))
        self._ran = False

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            C.lib().lk_dts_destroy(h)
            self._h = None

    @property
    def branching_pattern(self) -> np.ndarray:
        return self._bp.copy()

    def run(self, thres_neigh: int = 10) -> None:
        with D.torch().cuda.device(self._device):
            C.check(C.lib().lk_dts_run(self._h, int(thres_neigh), D.stream_ptr(self._device)))
        self._ran = True

    def transitions(self) -> int:
        """Transitions the last run simulated (each: ntrials H0 and ntrials H1
        folds built and scored)."""
        n = ctypes.c_uint64()
        C.check(C.lib().lk_dts_transitions(self._h, ctypes.byref(n)))
        return n.value

    def get_states(self) -> np.ndarray:
        """States [nstages * nthresholds * nprobs] (the reference's flat layout)."""
        n = self.nstages * self.nthresholds * self.nprobs
        out = np.zeros(n, STATE_DTYPE)
        C.check(C.lib().lk_dts_states(self._h, out.ctypes.data, n))
        return out

    def get_best_path_thresholds(self, min_pd: float = 0.1) -> np.ndarray:
        out = np.zeros(self.nstages, np.float32)
        n = ctypes.c_uint32()
        C.check(C.lib().lk_dts_best_path(self._h, float(min_pd), out.ctypes.data, ctypes.byref(n)))
        return out[: n.value].copy()

    def save(self, outdir: str = "./") -> str:
        """The reference's HDF5 file as ``.npz`` (same name stem and datasets)."""
        import os

        os.makedirs(outdir, exist_ok=True)
        name = (f"dynscheme_nstages_{self.nstages:03d}_nthresh_{self.nthresholds:03d}_nprobs_{self.nprobs:03d}_"
                f"snr_{float(self.thresholds[-1]):04.1f}.npz")
        path = os.path.join(outdir, name)
        np.savez(path, branching_pattern=self._bp, profile=self.profile, thresholds=self.thresholds,
                 probs=self.probs, guess_path=self.guess_path,
                 states=self.get_states().reshape(self.nstages, self.nthresholds, self.nprobs))
        return path


def dts_plan(branching_pattern, ref_ducy: float, nbins: int = 64, nprobs: int = 10, prob_min: float = 0.05,
             snr_final: float = 8.0, nthresholds: int = 100, ducy_max: float = 0.3, wtsp: float = 1.0,
             trials_start: int = 1) -> dict:
    """Host-only set-up of a scheme (no device): profile, thresholds, probs,
    guess path and box widths."""
    bp = np.ascontiguousarray(branching_pattern, dtype=np.float32)
    cfg = _DtsConfig(bp.ctypes.data, bp.size, float(ref_ducy), int(nbins), 1, int(nprobs), float(prob_min),
                     float(snr_final), int(nthresholds), float(ducy_max), float(wtsp), 0.7, int(trials_start), 0)
    out = {"profile": np.zeros(nbins, np.float32), "thresholds": np.zeros(nthresholds, np.float32),
           "probs": np.zeros(nprobs, np.float32), "guess_path": np.zeros(bp.size, np.float32),
           "widths": np.zeros(32, np.uint32)}
    nw = ctypes.c_uint32()
    C.check(C.lib().lk_dts_plan(ctypes.byref(cfg), out["profile"].ctypes.data, out["thresholds"].ctypes.data,
                                out["probs"].ctypes.data, out["guess_path"].ctypes.data, out["widths"].ctypes.data,
                                ctypes.byref(nw)))
    out["widths"] = out["widths"][: nw.value].copy()
    return out


def normal_lut() -> np.ndarray:
    """The generator's table of normal quantiles (2^17 + 1 floats)."""
    out = np.zeros((1 << 17) + 1, np.float32)
    C.check(C.lib().lk_dts_normal_lut(out.ctypes.data, out.size))
    return out
