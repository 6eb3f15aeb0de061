"""``FFAPlanTime``: FFA plan geometry, mirroring ``libloki.plans.FFAPlanTime``
(reference: include/loki/common/plans.hpp, lib/plans.cpp, bound at
src/loki_python.cpp:383-479 and src/loki_templates.hpp:23-44).

The geometry is computed by the native plan code (host). Coordinate tables
are resolved on the GPU by the same kernels the FFA uses and copied back.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as C
from . import _device as D
from .configs import PulsarSearchConfig

COORD_FREQ_DTYPE = np.dtype([("idx", np.uint32), ("shift", np.float32)])
COORD_DTYPE = np.dtype(
    [("i_tail", np.uint32), ("shift_tail", np.float32), ("i_head", np.uint32), ("shift_head", np.float32)]
)


def _strides(counts) -> np.ndarray:
    # FFAPlanBase::Impl::calculate_strides (lib/plans.cpp:334-343).
    n = len(counts)
    s = np.ones(n, dtype=np.uint64)
    for i in range(n - 2, -1, -1):
        s[i] = s[i + 1] * counts[i + 1]
    return s


class FFAPlanTime:
    """Time-domain FFA plan (``FFAPlan<float>``)."""

    def __init__(self, cfg: PulsarSearchConfig):
        self._cfg = cfg
        self._info = cfg._info
        self._handle = cfg._plan_handle

    @property
    def config(self) -> PulsarSearchConfig:
        return self._cfg

    @property
    def n_params(self) -> int:
        return int(self._info.nparams)

    @property
    def n_levels(self) -> int:
        return int(self._info.n_levels)

    def _levels(self, field, dtype) -> np.ndarray:
        return np.array(getattr(self._info, field)[: self.n_levels], dtype=dtype)

    @property
    def segment_lens(self) -> np.ndarray:
        return self._levels("segment_lens", np.uint64)

    @property
    def nsegments(self) -> np.ndarray:
        return self._levels("nsegments", np.uint64)

    @property
    def tsegments(self) -> np.ndarray:
        return self._levels("tsegments", np.float64)

    @property
    def ncoords(self) -> np.ndarray:
        return self._levels("ncoords", np.uint64)

    @property
    def ncoords_lb(self) -> np.ndarray:
        nc = self.ncoords.astype(np.float32)
        return np.where(nc > 0, np.log2(np.maximum(nc, 1)), 0).astype(np.float32)

    @property
    def ncoords_offsets(self) -> np.ndarray:
        return np.array(self._info.ncoords_offsets[: self.n_levels + 1], dtype=np.uint32)

    @property
    def param_counts(self) -> list[np.ndarray]:
        return [np.array(self._info.param_counts[l][: self.n_params], dtype=np.uint64) for l in range(self.n_levels)]

    @property
    def param_cart_strides(self) -> list[np.ndarray]:
        return [_strides(c) for c in self.param_counts]

    @property
    def dparams(self) -> list[np.ndarray]:
        return [np.array(self._info.dparams[l][: self.n_params]) for l in range(self.n_levels)]

    @property
    def dparams_actual(self) -> list[np.ndarray]:
        return [np.array(self._info.dparams_actual[l][: self.n_params]) for l in range(self.n_levels)]

    @property
    def coord_size(self) -> int:
        return int(self._info.coord_size)

    @property
    def coord_memory_usage(self) -> float:
        elem = 8 if self.n_params == 1 else 16
        return float(np.float32(self.coord_size * elem) / np.float32(1 << 30))

    @property
    def fold_shapes(self) -> list[np.ndarray]:
        shapes = []
        for l in range(self.n_levels):
            shapes.append(
                np.array([self.nsegments[l], *self.param_counts[l], 2, self._info.nbins], dtype=np.uint64)
            )
        return shapes

    @property
    def brute_fold_size(self) -> int:
        return int(self._info.brute_fold_size)

    @property
    def fold_size(self) -> int:
        return int(self._info.fold_size)

    @property
    def fold_size_time(self) -> int:
        return self.fold_size

    @property
    def buffer_size(self) -> int:
        return int(self._info.buffer_size)

    @property
    def buffer_size_time(self) -> int:
        return self.buffer_size

    @property
    def buffer_memory_usage(self) -> float:
        return float(np.float32(2 * self.buffer_size * 4) / np.float32(1 << 30))

    @property
    def score_widths(self) -> np.ndarray:
        return np.array(self._info.widths[: self._info.n_widths], dtype=np.uint64)

    def compute_param_grid(self, ffa_level: int) -> list[np.ndarray]:
        out = []
        for i in range(self.n_params):
            n = int(self._info.param_counts[ffa_level][i])
            g = np.zeros(n, dtype=np.float64)
            C.check(C.lib().lk_plan_param_grid(self._handle, ffa_level, i, g.ctypes.data, n))
            out.append(g)
        return out

    @property
    def param_grid(self) -> list[list[np.ndarray]]:
        return [self.compute_param_grid(l) for l in range(self.n_levels)]

    @property
    def params_dict(self) -> dict[str, np.ndarray]:
        grid = self.compute_param_grid(self.n_levels - 1)
        return dict(zip(self._cfg.param_names, grid))

    def _resolve(self, device_id: int = 0) -> np.ndarray:
        D.require_cuda(device_id)
        t = D.torch()
        dtype = COORD_FREQ_DTYPE if self.n_params == 1 else COORD_DTYPE
        nbytes = self.coord_size * dtype.itemsize
        buf = t.empty(nbytes, dtype=t.uint8, device=f"cuda:{device_id}")
        with t.cuda.device(device_id):
            C.check(C.lib().lk_plan_resolve_coords(self._handle, buf.data_ptr(), self.coord_size,
                                                   D.stream_ptr(device_id)))
            host = buf.cpu().numpy()
        return host.view(dtype)

    def _split(self, flat: np.ndarray) -> list[np.ndarray]:
        off = self.ncoords_offsets
        return [flat[off[l] : off[l + 1]].copy() for l in range(self.n_levels)]

    def resolve_coordinates(self, device_id: int = 0) -> list[np.ndarray]:
        if self.n_params < 2:
            raise RuntimeError(
                "resolve_coordinates only supports nparams>=2. For frequency coordinates, "
                "use resolve_coordinates_freq() instead."
            )
        return self._split(self._resolve(device_id))

    def resolve_coordinates_freq(self, device_id: int = 0) -> list[np.ndarray]:
        if self.n_params != 1:
            raise RuntimeError("resolve_coordinates_freq() only supports nparams=1")
        return self._split(self._resolve(device_id))

    def resolve_coordinates_flat(self, device_id: int = 0) -> np.ndarray:
        """All levels in one array (coord_size entries, level 0 zeroed)."""
        return self._resolve(device_id)


class FFAPlanFourier(FFAPlanTime):
    """FFAPlan<ComplexType> (reference ``libloki.plans.FFAPlanFourier``): the
    same levels and coordinates, folds of nbins_f = nbins // 2 + 1 complex
    harmonics; the *_time sizes are those of the fold back in time."""

    @property
    def nbins_f(self) -> int:
        return int(self._info.nbins) // 2 + 1

    def _fourier_size(self, time_size: int) -> int:
        return time_size // int(self._info.nbins) * self.nbins_f

    @property
    def fold_shapes(self) -> list[np.ndarray]:
        return [np.array([*s[:-1], self.nbins_f], dtype=np.uint64) for s in super().fold_shapes]

    @property
    def fold_shapes_time(self) -> list[np.ndarray]:
        return super().fold_shapes

    @property
    def brute_fold_size(self) -> int:
        return self._fourier_size(int(self._info.brute_fold_size))

    @property
    def fold_size(self) -> int:
        return self._fourier_size(int(self._info.fold_size))

    @property
    def fold_size_time(self) -> int:
        return int(self._info.fold_size)

    @property
    def buffer_size(self) -> int:
        return self._fourier_size(int(self._info.buffer_size))

    @property
    def buffer_size_time(self) -> int:
        return 2 * self.buffer_size

    @property
    def buffer_memory_usage(self) -> float:
        return float(np.float32(2 * self.buffer_size * 8) / np.float32(1 << 30))


# The reference binds the region planner in the plans submodule.
from .sweep import FFARegionPlannerFourier, FFARegionPlannerTime, generate_ffa_regions  # noqa: E402
