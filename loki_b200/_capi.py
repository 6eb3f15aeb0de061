"""ctypes binding of ``libloki_b200.so`` (the C ABI in ``include/loki_b200.h``).

The shared library is built in-tree (``make -C loki_b200/csrc``); importing this
module without it raises ``ImportError`` -- there is no fallback path.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libloki_b200.so")

LK_OK = 0
LK_ERR_INVALID_ARG = 1
LK_ERR_OOM = 2
LK_ERR_CUDA = 3
LK_ERR_DEVICE_TIMEOUT = 4
LK_ERR_UNSUPPORTED = 5
LK_ERR_INTERNAL = 6

LK_FP32, LK_BF16, LK_FP16 = 0, 1, 2
LK_SCORE_PER_WIDTH, LK_SCORE_MAX = 0, 1

LK_MAX_PARAMS = 5
LK_MAX_WIDTHS = 32
LK_MAX_LEVELS = 40

u64 = ctypes.c_uint64
u32 = ctypes.c_uint32
i32 = ctypes.c_int
f64 = ctypes.c_double
f32 = ctypes.c_float
vp = ctypes.c_void_p


class LokiError(RuntimeError):
    """Raised for a failed library call; ``status`` is the lk_status code.

    The reference raises ``RuntimeError`` (its DetailedException derives from
    std::runtime_error), so this subclasses it.
    """

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class LkConfig(ctypes.Structure):
    _fields_ = [
        ("nsamps", u64),
        ("tsamp", f64),
        ("nbins", u64),
        ("eta", f64),
        ("nparams", u32),
        ("param_limits", f64 * (2 * LK_MAX_PARAMS)),
        ("ducy_max", f64),
        ("wtsp", f64),
        ("bseg_brute", u64),
        ("bseg_ffa", u64),
        ("snr_min", f64),
        ("n_score_widths", u32),
        ("score_widths", u32 * LK_MAX_WIDTHS),
    ]


class LkPlanInfo(ctypes.Structure):
    _fields_ = [
        ("nparams", u32),
        ("n_levels", u32),
        ("nsamps", u64),
        ("nbins", u64),
        ("tsamp", f64),
        ("bseg_brute", u64),
        ("bseg_ffa", u64),
        ("tseg_brute", f64),
        ("tseg_ffa", f64),
        ("segment_lens", u64 * LK_MAX_LEVELS),
        ("nsegments", u64 * LK_MAX_LEVELS),
        ("tsegments", f64 * LK_MAX_LEVELS),
        ("ncoords", u64 * LK_MAX_LEVELS),
        ("ncoords_offsets", u32 * (LK_MAX_LEVELS + 1)),
        ("param_counts", (u64 * LK_MAX_PARAMS) * LK_MAX_LEVELS),
        ("dparams", (f64 * LK_MAX_PARAMS) * LK_MAX_LEVELS),
        ("dparams_actual", (f64 * LK_MAX_PARAMS) * LK_MAX_LEVELS),
        ("buffer_size", u64),
        ("fold_size", u64),
        ("brute_fold_size", u64),
        ("coord_size", u64),
        ("n_widths", u32),
        ("widths", u32 * LK_MAX_WIDTHS),
        ("snr_min", f64),
    ]


STAGE_NAMES = {0: "interleave", 1: "brute_fold", 2: "merge", 3: "merge_score", 4: "compact", 5: "rescore",
               6: "transform", 7: "score"}


class LkStageTime(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("level", ctypes.c_int32), ("launches", u32), ("ms", f32),
                ("bytes", u64)]


class LkTuning(ctypes.Structure):
    _fields_ = [("bf_rows", u32), ("bf_warps", u32), ("bf_stages", u32), ("merge_rows_in_flight", ctypes.c_int32),
                ("score_cells_per_block", u32), ("candidates", u32), ("bf_ms", f32), ("merge_ms", f32),
                ("score_ms", f32), ("bf_tmem_warps", u32)]


class LkSweepOptions(ctypes.Structure):
    _fields_ = [("max_memory_gb", f64), ("octave_scale", f64), ("nbins_max", u64),
                ("max_passing_candidates", u64), ("decode_chunk_widths", ctypes.c_int32),
                ("device_memory_model", ctypes.c_int32), ("executor_mode", ctypes.c_int32),
                ("autotune", ctypes.c_int32), ("use_fourier", ctypes.c_int32), ("nbins_min_lossy_bf", u64),
                ("plan_sizes", ctypes.c_int32)]


class LkSweepChunk(ctypes.Structure):
    _fields_ = [("f_min", f64), ("f_max", f64), ("nominal_f_start", f64), ("nominal_f_end", f64),
                ("nbins", u64), ("eta", f64), ("buffer_size", u64), ("coord_size", u64), ("ncoords", u64),
                ("n_levels", u64), ("memory_gb", f64), ("allocated_gb", f64)]


# (name, restype, argtypes) of every exported entry point, in header order.
class LkPruneStats(ctypes.Structure):
    _fields_ = [
        ("level", u64),
        ("seg_idx", u64),
        ("n_branches", u64),
        ("n_leaves", u64),
        ("n_leaves_phy", u64),
        ("n_leaves_surv", u64),
        ("threshold", f32),
        ("score_min", f32),
        ("score_max", f32),
        ("pad", f32),
    ]


SIGNATURES = [
    ("lk_last_error", ctypes.c_char_p, []),
    ("lk_version", i32, []),
    ("lk_plan_create", i32, [vp, vp]),
    ("lk_plan_destroy", None, [vp]),
    ("lk_plan_get_info", i32, [vp, vp]),
    ("lk_plan_param_grid", i32, [vp, u32, u32, vp, u64]),
    ("lk_plan_dparams", i32, [vp, f64, i32, vp]),
    ("lk_plan_resolve_coords", i32, [vp, vp, u64, vp]),
    ("lk_ffa_create", i32, [vp, i32, i32, vp]),
    ("lk_ffa_destroy", None, [vp]),
    ("lk_ffa_workspace_bytes", i32, [vp, vp]),
    ("lk_ffa_execute", i32, [vp, vp, vp, vp, u64, vp]),
    ("lk_ffa_scores", i32, [vp, vp, vp, vp, u64, vp]),
    ("lk_ffa_search", i32, [vp, vp, vp, f32, vp, vp, u64, vp, vp]),
    ("lk_fourier_create", i32, [vp, i32, u64, vp]),
    ("lk_fourier_destroy", None, [vp]),
    ("lk_fourier_info", i32, [vp, vp, vp, vp, vp, vp]),
    ("lk_fourier_execute", i32, [vp, vp, vp, vp, u64, vp]),
    ("lk_fourier_execute_time", i32, [vp, vp, vp, vp, u64, vp]),
    ("lk_fourier_scores", i32, [vp, vp, vp, vp, u64, vp]),
    ("lk_fourier_search", i32, [vp, vp, vp, f32, vp, vp, u64, vp, vp]),
    ("lk_fourier_set_profiling", i32, [vp, i32]),
    ("lk_fourier_set_level0", i32, [vp, i32]),
    ("lk_fourier_get_level0", i32, [vp, vp]),
    ("lk_fourier_autotune", i32, [vp, vp, vp, u32, vp, vp]),
    ("lk_fourier_status", i32, [vp, vp, vp]),
    ("lk_fourier_get_profile", i32, [vp, vp, vp, u32, vp]),
    ("lk_fourier_brute_fold", i32, [vp, vp, u64, vp, u64, u64, u64, f64, f64, vp, u64, i32, vp]),
    ("lk_ffa_create_batched", i32, [vp, i32, i32, u64, vp]),
    ("lk_ffa_execute_batch", i32, [vp, vp, vp, u64, vp, u64, vp]),
    ("lk_ffa_scores_batch", i32, [vp, vp, vp, u64, vp, u64, vp]),
    ("lk_ffa_search_batch", i32, [vp, vp, vp, u64, f32, vp, vp, u64, vp, vp]),
    ("lk_ffa_set_batch_lengths", i32, [vp, vp]),
    ("lk_ffa_status", i32, [vp, vp, vp]),
    ("lk_ffa_set_rescore_margin", i32, [vp, ctypes.c_float, ctypes.c_float]),
    ("lk_ffa_get_rescore_margin", i32, [vp, vp, vp]),
    ("lk_ffa_rescored_cells", i32, [vp, vp, vp]),
    ("lk_sweep_create", i32, [vp, vp, i32, i32, vp]),
    ("lk_sweep_destroy", None, [vp]),
    ("lk_sweep_nchunks", i32, [vp, vp]),
    ("lk_sweep_chunk_info", i32, [vp, u64, vp]),
    ("lk_sweep_execute", i32, [vp, vp, vp, vp]),
    ("lk_sweep_results", i32, [vp, vp, vp, u64, vp, vp]),
    ("lk_sweep_set_profiling", i32, [vp, i32]),
    ("lk_sweep_get_profile", i32, [vp, vp, u32, vp]),
    ("lk_generate_ffa_regions", i32, [f64, f64, f64, u64, f64, f64, u64, vp, u64, vp]),
    ("lk_ffa_autotune", i32, [vp, vp, vp, u32, vp, vp]),
    ("lk_ffa_get_tuning", i32, [vp, vp]),
    ("lk_ffa_set_tuning", i32, [vp, vp]),
    ("lk_ffa_set_profiling", i32, [vp, i32]),
    ("lk_ffa_get_profile", i32, [vp, vp, vp, u32, vp]),
    ("lk_brute_fold_create", i32, [vp, u64, u64, u64, u64, f64, f64, i32, vp]),
    ("lk_brute_fold_destroy", None, [vp]),
    ("lk_brute_fold_execute", i32, [vp, vp, vp, vp, vp]),
    ("lk_box_width_trials", i32, [u64, f64, f64, vp, u32, vp]),
    ("lk_snr_boxcar_3d", i32, [vp, u64, u32, vp, u32, i32, vp, vp]),
    ("lk_snr_boxcar_2d_max", i32, [vp, u64, u32, vp, u32, f32, vp, vp]),
    ("lk_compact_scratch_bytes", u64, [u64]),
    ("lk_compact_ge", i32, [vp, u64, f32, vp, vp, u64, vp, vp, vp]),
    ("lk_compact_ge_noalloc", i32, [vp, u64, f32, vp, vp, u64, vp, vp]),
    ("lk_mc_create", i32, [u64, u32, vp, u32, i32, vp]),
    ("lk_mc_destroy", None, [vp]),
    ("lk_mc_stage", i32, [vp, vp, u64, vp, u64, vp, u64, vp, i32, f32, vp, f32, f32, f32, vp, u32, vp, vp, vp,
                          vp, vp, vp, vp]),
    ("lk_mc_status", i32, [vp, vp, vp]),
    ("lk_prune_create", i32, [vp, u64, u64, u64, i32, i32, vp]),
    ("lk_prune_destroy", None, [vp]),
    ("lk_plan_branching_pattern", i32, [vp, u64, i32, vp, u64, vp]),
    ("lk_prune_set_tail", i32, [vp, i32]),
    ("lk_prune_run_many", i32, [vp, u64, vp, vp, vp, u64, u64, vp, u64, vp, vp]),
    ("lk_prune_run", i32, [vp, vp, u64, vp, u64, u64, vp, u64, vp, vp]),
    ("lk_prune_finalize", i32, [vp, vp, vp]),
    ("lk_prune_get_scores_ep", i32, [vp, vp, u64, vp]),
    ("lk_prune_tree_size", i32, [vp, vp]),
    ("lk_prune_get_tree", i32, [vp, vp, vp, vp, u64, vp]),
    ("lk_taylor_seed", i32, [vp, vp, vp]),
    ("lk_taylor_branch", i32, [vp, vp, u64, f64, u64, vp, vp, u64, vp, vp]),
    ("lk_taylor_resolve", i32, [vp, vp, u64, vp, vp, vp, vp]),
    ("lk_taylor_transform", i32, [vp, vp, u64, vp, u64, f64, f64, i32, vp]),
    ("lk_prune_create_basis", i32, [vp, u64, u64, u64, i32, i32, i32, vp]),
    ("lk_plan_branching_pattern_basis", i32, [vp, u64, i32, i32, vp, u64, vp]),
    ("lk_taylor_to_cheby", i32, [vp, u64, u32, f64, vp]),
    ("lk_cheby_to_taylor", i32, [vp, u64, u32, f64, vp]),
    ("lk_cheby_branch", i32, [vp, vp, u64, f64, f64, f64, f64, u64, vp, vp, u64, vp, vp]),
    ("lk_cheby_resolve", i32, [vp, vp, u64, vp, vp, vp, vp]),
    ("lk_cheby_transform", i32, [vp, vp, u64, vp, u64, f64, f64, f64, f64, vp]),
    ("lk_shift_add_batch", i32, [vp, vp, vp, u64, vp, vp, vp, u32, u64, u64, u64, vp]),
    ("lk_score_filter", i32, [vp, u64, u32, vp, u32, f32, vp, vp, vp, vp]),
    ("lk_wait_check", i32, [u32, i32, vp, vp]),
    ("lk_dts_create", i32, [vp, i32, vp]),
    ("lk_dts_destroy", None, [vp]),
    ("lk_dts_run", i32, [vp, u32, vp]),
    ("lk_dts_info", i32, [vp, vp, vp, vp, vp, vp]),
    ("lk_dts_arrays", i32, [vp, vp, vp, vp, vp, vp]),
    ("lk_dts_states", i32, [vp, vp, u64]),
    ("lk_dts_best_path", i32, [vp, f32, vp, vp]),
    ("lk_dts_normal_lut", i32, [vp, u64]),
    ("lk_dts_plan", i32, [vp, vp, vp, vp, vp, vp, vp]),
    ("lk_dts_transitions", i32, [vp, vp]),
]

_lib: ctypes.CDLL | None = None


def lib() -> ctypes.CDLL:
    """The loaded native library (loaded once)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"loki_b200 native library not found at {LIB_PATH}; build it with "
                "`make -C loki_b200/csrc` (or __graft_entry__.build())"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != LK_OK:
        msg = lib().lk_last_error().decode(errors="replace")
        if rc == LK_ERR_OOM:
            raise MemoryError(msg)
        raise LokiError(rc, msg)


# Fail loudly when a computing module is imported without the native library.
lib()
