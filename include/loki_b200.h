/* loki_b200: B200-native (sm_100a) FFA folding, boxcar scoring and pruning
 * leaf step for pulsar searches, behind a plain C ABI.
 *
 * Conventions
 *   - Every entry point returns int: LK_OK (0) or an lk_status code; the
 *     message of the last failure on the calling thread is lk_last_error().
 *   - Device buffers (d_*) are owned by the caller. Objects (lk_plan, lk_ffa,
 *     lk_brute_fold) own their device tables and scratch.
 *   - Work is enqueued on the given stream (cudaStream_t passed as
 *     lk_stream_t; NULL is the legacy default stream). Entry points named
 *     *_execute / *_scores / *_search do not synchronise the stream.
 *   - A plan is immutable after creation; an executor is used by one stream
 *     at a time.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   lk_plan_*         plans::FFAPlan<float>, search::PulsarSearchConfig
 *                     (include/loki/common/plans.hpp:21-140,
 *                      include/loki/search/configs.hpp:22-164)
 *   lk_ffa_*          algorithms::FFACUDA<float> (include/loki/algorithms/ffa.hpp:100-153),
 *                     compute_ffa_cuda / compute_ffa_scores_cuda (lib/ffa_cuda.cu:609-650)
 *   lk_brute_fold_*   algorithms::BruteFoldCUDA<float> (include/loki/algorithms/fold.hpp:78-134)
 *   lk_snr_boxcar_*   detection::snr_boxcar_{3d,3d_max,2d_max}_cuda (lib/score_cuda.cu:253-513)
 *   lk_compact_ge     score compaction of FFAFreqSweep (lib/ffa_freq_sweep.cpp:182-195)
 *   lk_prune_*        PruneImpl / EPMultiPass per ref_seg run (lib/prune.cpp:40-226,429-620)
 *                     and PruneCUDA (include/loki/algorithms/prune.hpp)
 *   lk_taylor_*, lk_shift_add_batch, lk_score_filter
 *                     the Taylor PruneDPFuncts steps (include/loki/core/dynamic.hpp:22-115):
 *                     core::poly_taylor_{seed,branch,resolve,transform}_batch
 *                     (include/loki/core/taylor.hpp:16-79), kernels::shift_add_linear_batch
 *                     (lib/loki/kernels.hpp:100), detection::score_and_filter_max_with_cache
 *                     (include/loki/detection/score.hpp:113-119)
 *   lk_mc_*           simulate_score_prune_fused of DynamicThresholdScheme
 *                     (lib/thresholds.cpp:358-431)
 */
#ifndef LOKI_B200_H
#define LOKI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* lk_stream_t;

enum lk_status {
    LK_OK = 0,
    LK_ERR_INVALID_ARG = 1,   /* argument/config rejected (reference throws invalid_argument/runtime_error) */
    LK_ERR_OOM = 2,           /* device or host allocation failed */
    LK_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    LK_ERR_DEVICE_TIMEOUT = 4,/* a bounded device-side wait gave up (status word set) */
    LK_ERR_UNSUPPORTED = 5,   /* valid request outside what this build implements */
    LK_ERR_INTERNAL = 6
};

/* Storage type of intermediate fold levels. Accumulation is always FP32. */
enum lk_dtype { LK_FP32 = 0, LK_BF16 = 1, LK_FP16 = 2 };

enum lk_score_mode { LK_SCORE_PER_WIDTH = 0, LK_SCORE_MAX = 1 };

#define LK_MAX_PARAMS 5
#define LK_MAX_WIDTHS 32
#define LK_MAX_LEVELS 40

/* Search configuration: the PulsarSearchConfig fields the FFA path reads
 * (include/loki/search/configs.hpp:25-47). param_limits holds nparams
 * (min, max) pairs ordered (..., jerk, accel, freq). bseg_brute / bseg_ffa of
 * 0 select the reference defaults (lib/configs.cpp:295-302).
 * n_score_widths == 0 selects generate_box_width_trials(nbins, ducy_max, wtsp)
 * (lib/score.cpp:390-405); otherwise score_widths[0..n) are used as given. */
typedef struct lk_config {
    uint64_t nsamps;
    double tsamp;
    uint64_t nbins;
    double eta;
    uint32_t nparams;
    double param_limits[2 * LK_MAX_PARAMS];
    double ducy_max;
    double wtsp;
    uint64_t bseg_brute;
    uint64_t bseg_ffa;
    double snr_min;
    uint32_t n_score_widths;
    uint32_t score_widths[LK_MAX_WIDTHS];
} lk_config;

/* Plan geometry (FFAPlanBase getters, include/loki/common/plans.hpp:38-78). */
typedef struct lk_plan_info {
    uint32_t nparams;
    uint32_t n_levels;
    uint64_t nsamps;
    uint64_t nbins;
    double tsamp;
    uint64_t bseg_brute;
    uint64_t bseg_ffa;
    double tseg_brute;
    double tseg_ffa;
    uint64_t segment_lens[LK_MAX_LEVELS];
    uint64_t nsegments[LK_MAX_LEVELS];
    double tsegments[LK_MAX_LEVELS];
    uint64_t ncoords[LK_MAX_LEVELS];
    uint32_t ncoords_offsets[LK_MAX_LEVELS + 1];
    uint64_t param_counts[LK_MAX_LEVELS][LK_MAX_PARAMS];
    double dparams[LK_MAX_LEVELS][LK_MAX_PARAMS];
    double dparams_actual[LK_MAX_LEVELS][LK_MAX_PARAMS];
    uint64_t buffer_size;     /* FFAPlan::get_buffer_size (lib/plans.cpp:463-470) */
    uint64_t fold_size;       /* final level [nseg, counts..., 2, nbins] */
    uint64_t brute_fold_size; /* level 0 */
    uint64_t coord_size;      /* sum of ncoords over levels */
    uint32_t n_widths;
    uint32_t widths[LK_MAX_WIDTHS];
    double snr_min;
} lk_plan_info;

typedef struct lk_plan lk_plan;
typedef struct lk_ffa lk_ffa;
typedef struct lk_brute_fold lk_brute_fold;
typedef struct lk_fourier lk_fourier;

/* ---- library ---------------------------------------------------------- */
const char* lk_last_error(void);
int lk_version(void);

/* ---- plan (host only; no device work) ---------------------------------- */
/* Replaces FFAPlan<float>(PulsarSearchConfig(...)) (lib/plans.cpp:33-36,264-333,
 * lib/configs.cpp:16-95). */
int lk_plan_create(const lk_config* cfg, lk_plan** out);
void lk_plan_destroy(lk_plan* plan);
int lk_plan_get_info(const lk_plan* plan, lk_plan_info* out);
/* Cell centres of one parameter at one level: psr_utils::range_param
 * (lib/loki/psr_utils.hpp:254-270), as FFAPlanBase::compute_param_grid
 * (lib/plans.cpp:152-162). Writes min(n, count) values. */
int lk_plan_param_grid(const lk_plan* plan, uint32_t level, uint32_t iparam, double* out,
                       uint64_t n);
/* Grid steps for a segment of length tseg_cur seconds, nparams values:
 * kind 0 = PulsarSearchConfig::get_dparams, 1 = get_dparams_f,
 * 2 = get_dparams_actual (lib/configs.cpp:152-174). */
int lk_plan_dparams(const lk_plan* plan, double tseg_cur, int kind, double* out);

/* Resolve the coordinate tables of every level on the device, in the
 * reference layout (FFACoordFreq {u32 idx; f32 shift} when nparams == 1,
 * FFACoord {u32 i_tail; f32 shift_tail; u32 i_head; f32 shift_head}
 * otherwise), coord_size entries, level 0 zeroed. Replaces
 * FFAPlanBase::resolve_coordinates[_freq] (lib/plans.cpp:64-132). */
int lk_plan_resolve_coords(const lk_plan* plan, void* d_coords, uint64_t n_coords,
                           lk_stream_t stream);

/* ---- FFA executor (replaces FFACUDA<float>) ---------------------------- */
/* Builds the device tables (coordinates, brute-fold run tables) and scratch
 * for `plan` on `device`. storage: lk_dtype of intermediate levels.
 * LK_FP32: every level FP32 (the reference's FFACUDA<float>).
 * LK_BF16: levels 1 .. L-2 stored as BF16, every add FP32; level 0 stays
 *   FP32. Folds and scores then carry BF16 rounding error; lk_ffa_search
 *   rescores every final cell within a margin of snr_min exactly (from the
 *   FP32 level 0, same add tree) so its candidate set and S/N values are the
 *   LK_FP32 ones. At most 8192 level-0 segments.
 * LK_FP16: rejected (LK_ERR_UNSUPPORTED): V rows outgrow FP16's range. */
int lk_ffa_create(const lk_plan* plan, int device, int storage, lk_ffa** out);
void lk_ffa_destroy(lk_ffa* ffa);
/* Device bytes owned by the executor. */
int lk_ffa_workspace_bytes(const lk_ffa* ffa, uint64_t* bytes);
/* Final-level fold, FP32, fold_size floats. Replaces FFACUDA::execute
 * (lib/ffa_cuda.cu:171-196). */
int lk_ffa_execute(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, float* d_fold,
                   uint64_t fold_len, lk_stream_t stream);
/* Boxcar S/N of every final coordinate and width, [ncoords, n_widths] FP32;
 * the final merge level and the score are one kernel (the final fold is not
 * written). Replaces compute_ffa_scores_cuda (lib/ffa_cuda.cu:630-650). */
int lk_ffa_scores(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, float* d_scores,
                  uint64_t scores_len, lk_stream_t stream);
/* Scores plus threshold compaction `score >= snr_min` in flat index order
 * (coord * n_widths + width), as FFAFreqSweep::execute_ffa_region
 * (lib/ffa_freq_sweep.cpp:182-195). Writes up to max_cands (index, S/N)
 * pairs and the total number passing to *d_count (which may exceed
 * max_cands; the kept entries are then the first max_cands in order). */
int lk_ffa_search(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, float snr_min,
                  uint32_t* d_idx, float* d_snr, uint64_t max_cands, uint64_t* d_count,
                  lk_stream_t stream);

/* Batched executor: nbatch <= max_batch series of the plan's nsamps samples,
 * stored back to back in d_ts_e / d_ts_v, folded and scored together (one
 * launch per level for the whole batch; a batch is, level by level, one series
 * with nbatch times the segments). Outputs are each series' single-series
 * output, back to back: folds [nbatch][fold_size], scores [nbatch][ncoords]
 * [nwidths], and search indices flat over [nbatch][ncoords][nwidths]
 * (nbatch * ncoords * nwidths < 2^32). Intermediate buffers are sized for
 * max_batch series. The single-series calls above are nbatch = 1. */
int lk_ffa_create_batched(const lk_plan* plan, int device, int storage, uint64_t max_batch,
                          lk_ffa** out);
int lk_ffa_execute_batch(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint64_t nbatch,
                         float* d_fold, uint64_t fold_len, lk_stream_t stream);
int lk_ffa_scores_batch(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint64_t nbatch,
                        float* d_scores, uint64_t scores_len, lk_stream_t stream);
int lk_ffa_search_batch(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint64_t nbatch,
                        float snr_min, uint32_t* d_idx, float* d_snr, uint64_t max_cands,
                        uint64_t* d_count, lk_stream_t stream);
/* Valid samples of each series of a batch, as a DEVICE array of uint64 (one
 * per series of the next batched calls; NULL turns it off). Every sample of
 * series i at or past d_lengths[i] must be zero: the brute fold then skips
 * the segments that hold none of the first d_lengths[i] samples (in groups
 * of 8) and sets their folds to +0.0, the result folding the zeros gives, so
 * outputs do not change. The array is read by every launch (a captured graph
 * sees lengths written into it later) and must outlive the calls. The
 * reference pads uneven series to a power of two (lib/configs.cpp:264); this
 * lets the padding cost nothing. */
int lk_ffa_set_batch_lengths(lk_ffa* ffa, const uint64_t* d_lengths);

/* ---- Fourier-domain FFA (replaces FFACUDA<ComplexTypeCUDA>) ------------- */
/* The FFA of the reference's use_fourier = true path (the default of
 * PulsarSearchConfig, include/loki/search/configs.hpp:32): folds are kept as
 * nbins_f = nbins / 2 + 1 complex harmonics, merges rotate them by the
 * coordinates' fractional shifts (lib/kernels.cpp:241-453, 942-1130), and
 * results return to time by an inverse real transform scaled by 1 / nbins
 * (lib/fft.cpp:503-552). Level 0 is the direct transform of each segment
 * (lib/kernels.cpp:1156-1242) for nbins <= nbins_min_lossy_bf, else the
 * time-domain brute fold followed by a real transform (lib/ffa.cpp:170-240).
 * nbins_min_lossy_bf 0 selects the reference default 64. Complex arrays are
 * interleaved (re, im) FP32, as cuda::std::complex<float>. FP32 sums; phases
 * reduced modulo one cycle in FP64 before the FP32 sine and cosine. */
/* BruteFoldCUDA<ComplexTypeCUDA> / compute_brute_fold_cuda<ComplexTypeCUDA>
 * (lib/fold_cuda.cu, lib/kernels_cuda.cu:856-965): the direct transform of
 * each segment at each frequency, [nsamps / segment_len, nfreqs, 2,
 * nbins / 2 + 1] complex (fold_len counts complex values). freqs is a host
 * array. */
int lk_fourier_brute_fold(const float* d_ts_e, const float* d_ts_v, uint64_t nsamps,
                          const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                          uint64_t nbins, double tsamp, double t_ref, float* d_fold,
                          uint64_t fold_len, int device, lk_stream_t stream);
int lk_fourier_create(const lk_plan* plan, int device, uint64_t nbins_min_lossy_bf,
                      lk_fourier** out);
void lk_fourier_destroy(lk_fourier* f);
/* Kernel of the level-0 direct transform (results agree to FP32 accuracy):
 * AUTO = the tensor cores when the shape allows (nbins / 2 <= 64 harmonics,
 * segment length a multiple of 8), else the CUDA cores. */
enum lk_fourier_level0 {
    LK_FOURIER_L0_AUTO = 0,
    LK_FOURIER_L0_CUDA_CORES = 1,  /* FP32 phasor recurrence per harmonic */
    LK_FOURIER_L0_TENSOR_CORES = 2 /* tcgen05.mma, three FP16 hi / lo passes, FP32 sums */
};
int lk_fourier_set_level0(lk_fourier* f, int mode);
/* Level-0 kernel the executor runs now: LK_FOURIER_L0_CUDA_CORES or
 * LK_FOURIER_L0_TENSOR_CORES, or LK_FOURIER_L0_AUTO (0) for the lossy level 0
 * (time-domain brute fold + real transform). */
int lk_fourier_get_level0(const lk_fourier* f, int* mode);
/* Times the tensor-core level 0's tilings (column subtiles per block, K
 * part length) on these device series and keeps the fastest (synchronises the
 * stream; results agree to FP32 accuracy whichever is kept); *level0_ms the
 * kept time, 0 when level 0 is not on the tensor cores. No reference
 * counterpart (launch shapes). */
int lk_fourier_autotune(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, uint32_t reps,
                        float* level0_ms, lk_stream_t stream);
/* Synchronises the stream; the device status word (bounded-wait give-ups). */
int lk_fourier_status(lk_fourier* f, lk_stream_t stream, uint32_t* status);
/* nbins_f; final fold sizes (complex values, and floats back in time);
 * lossy = 1 when level 0 is the brute fold + real transform. */
int lk_fourier_info(const lk_fourier* f, uint64_t* nbins_f, uint64_t* fold_size,
                    uint64_t* fold_size_time, int* lossy, uint64_t* workspace_bytes);
/* FFACUDA<ComplexTypeCUDA>::execute(ts_e, ts_v, span<ComplexTypeCUDA>, stream)
 * (include/loki/algorithms/ffa.hpp:126-134): final complex fold
 * [nseg, ncoords, 2, nbins_f]; fold_len counts complex values. */
int lk_fourier_execute(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float* d_fold,
                       uint64_t fold_len, lk_stream_t stream);
/* FFACUDA<ComplexTypeCUDA>::execute(ts_e, ts_v, span<float>, stream)
 * (ffa.hpp:142-147): the final fold back in time, [nseg, ncoords, 2, nbins]
 * FP32 (fold_size_time floats). */
int lk_fourier_execute_time(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float* d_fold,
                            uint64_t fold_len, lk_stream_t stream);
/* compute_ffa_scores with use_fourier (lib/ffa.cpp:444-466): boxcar S/N of
 * every final coordinate and width of the fold back in time. */
int lk_fourier_scores(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float* d_scores,
                      uint64_t scores_len, lk_stream_t stream);
/* Scores plus threshold compaction, as lk_ffa_search. */
int lk_fourier_search(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float snr_min,
                      uint32_t* d_idx, float* d_snr, uint64_t max_cands, uint64_t* d_count,
                      lk_stream_t stream);

/* Synchronises the stream and reports the executor's device status word
 * (0 = no bounded wait gave up). */
int lk_ffa_status(lk_ffa* ffa, lk_stream_t stream, uint32_t* status);

/* LK_BF16 search margin (no reference counterpart): a search rescores every
 * final cell whose approximate best S/N is >= (snr_min - margin_abs) /
 * (1 + margin_rel). Defaults follow from the level count (12 standard
 * deviations of the BF16 rounding error plus a bound for the V rows). Both
 * must be finite and >= 0; calls on an LK_FP32 executor are no-ops. */
int lk_ffa_set_rescore_margin(lk_ffa* ffa, float margin_abs, float margin_rel);
int lk_ffa_get_rescore_margin(const lk_ffa* ffa, float* margin_abs, float* margin_rel);
/* ---- FFAFreqSweep (replaces algorithms::FFAFreqSweep) ------------------- */
/* The reference's production caller (lib/ffa_freq_sweep.cpp:76-269,
 * lib/regions.cpp:31-514): octave regions of growing nbins, each cut into
 * chunks that fit max_memory_gb (bisection over the chunk width, frequency
 * ranges widened by the largest Doppler drift), then per chunk FFA + boxcar
 * scores + `>= snr_min` compaction and the parameter decode of every passing
 * (coordinate, width). The base configuration supplies nsamps, tsamp, the
 * smallest nbins, eta, the parameter limits (frequency last), widths and
 * snr_min. Results replace the HDF5 writer: per candidate nparams + 1
 * doubles (parameter values, then the width) and its S/N, in region order. */
typedef struct lk_sweep lk_sweep;
typedef struct lk_sweep_options {
    double max_memory_gb;             /* max_process_memory_gb (reference default 8.0) */
    double octave_scale;              /* 2.0 */
    uint64_t nbins_max;               /* 1024 */
    uint64_t max_passing_candidates;  /* 1 << 22 */
    /* 0: decode every chunk's candidates with the base configuration's width
     * list, as save_results does (lib/ffa_freq_sweep.cpp:202-233), which
     * mislabels candidates of a chunk whose nbins gives another width count;
     * 1: decode with the chunk's own widths. */
    int32_t decode_chunk_widths;
    /* 1: the device memory model of FFAFreqSweepCUDA (input series, scores and
     * indices, fold buffers, coordinates; lib/regions.cpp:136-149); 0: the
     * process model of FFAFreqSweep (fold buffers, coordinates, scores,
     * indices, write batch; lib/regions.cpp:101-135). */
    int32_t device_memory_model;
    /* Chunk executors: 0 decides at the first execute (every chunk's executor
     * kept resident, chunks overlapping on two streams, when their planned
     * memory fits in free device memory with room to spare; else one chunk at
     * a time, each executor released after its chunk), 1 resident, 2 one at a
     * time. Results do not depend on it. */
    int32_t executor_mode;
    /* 1: time each chunk executor's launch shapes on the first execute's
     * series (lk_ffa_autotune) and keep them, also for executors re-created
     * in mode 2; results do not change. */
    int32_t autotune;
    /* 1: every chunk through the Fourier-domain FFA (lk_fourier_*), as
     * FFAFreqSweep does for use_fourier = true (lib/ffa_freq_sweep.cpp:
     * 273-281); the planner then sizes fold buffers in complex harmonics of
     * 8 bytes (FFAPlan<ComplexType>, lib/regions.cpp:111-115). */
    int32_t use_fourier;
    /* nbins above which a Fourier chunk's level 0 is the lossy one (0: 64). */
    uint64_t nbins_min_lossy_bf;
    /* Fold-buffer sizes of the plan: 0 as the executors need them (complex
     * harmonics with use_fourier, else nbins per row), 1 nbins per row
     * (FFARegionPlanner<float>), 2 nbins / 2 + 1 harmonics per row
     * (FFARegionPlanner<ComplexType>). Fold elements count 8 bytes with
     * use_fourier, else 4, whatever the sizes (lib/regions.cpp:111-115).
     * 1 and 2 are for planning only. */
    int32_t plan_sizes;
} lk_sweep_options;
/* regions::generate_ffa_regions (lib/regions.cpp:31-78): rows of (f_start,
 * f_end, nbins, eta); *n_out regions, rows written up to cap. */
int lk_generate_ffa_regions(double p_min, double p_max, double tsamp, uint64_t nbins_min,
                            double eta_min, double octave_scale, uint64_t nbins_max,
                            double* rows, uint64_t cap, uint64_t* n_out);
typedef struct lk_sweep_chunk {
    double f_min, f_max;              /* drift-widened frequency limits */
    double nominal_f_start, nominal_f_end;
    uint64_t nbins;
    double eta;
    uint64_t buffer_size, coord_size, ncoords, n_levels;
    double memory_gb;                 /* this chunk alone */
    double allocated_gb;              /* with the largest sizes of the chunks up to it */
} lk_sweep_chunk;
int lk_sweep_create(const lk_config* base, const lk_sweep_options* opt, int device, int storage,
                    lk_sweep** out);
void lk_sweep_destroy(lk_sweep* sw);
int lk_sweep_nchunks(const lk_sweep* sw, uint64_t* n);
int lk_sweep_chunk_info(const lk_sweep* sw, uint64_t i, lk_sweep_chunk* out);
/* Device series (nsamps floats each). Synchronises the stream. */
int lk_sweep_execute(lk_sweep* sw, const float* d_ts_e, const float* d_ts_v, lk_stream_t stream);
/* Host outputs of the last execute: *n_out candidates; params [n][nparams + 1]
 * and scores [n] written up to max_out; region_counts [nchunks] may be NULL. */
int lk_sweep_results(const lk_sweep* sw, double* params, float* scores, uint64_t max_out,
                     uint64_t* n_out, uint64_t* region_counts);

/* Launch-shape tuning (an autotuner of this library; no reference counterpart).
 * bf_*: brute fold rows (E, V) per consumer warp (1 or 2), consumer warps
 * per block (0: the wave-count rule), shared-memory ring depth in 32-sample
 * words; merge_rows_in_flight: output rows per warp whose loads are issued
 * together in a merge level (0: the default for nbins); score_cells_per_block:
 * final cells per block of the fused final level (0: the most that fit). */
typedef struct lk_tuning {
    uint32_t bf_rows;
    uint32_t bf_warps;
    uint32_t bf_stages;
    int32_t merge_rows_in_flight;
    uint32_t score_cells_per_block;
    uint32_t candidates; /* configurations lk_ffa_autotune timed */
    float bf_ms;         /* best median stage times (ms): brute fold (+ interleave), */
    float merge_ms;      /* all merge levels, */
    float score_ms;      /* fused final level */
    uint32_t bf_tmem_warps; /* brute fold: consumer warps (of bf_warps) whose sums are in tensor memory */
} lk_tuning;
/* Times the candidates on the given device series (one search's inputs;
 * reps timed passes each, median) and keeps the fastest shape of each stage.
 * Results of every later call are unchanged (same sums, same order).
 * Synchronises the stream. A plan that stops at several segments (the
 * pruning input, bseg_ffa) has no fused final level: its brute fold and
 * merges are tuned and score_ms is 0. */
int lk_ffa_autotune(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint32_t reps,
                    lk_tuning* out, lk_stream_t stream);
int lk_ffa_get_tuning(const lk_ffa* ffa, lk_tuning* out);
/* Applies a saved tuning (validated against the plan). */
int lk_ffa_set_tuning(lk_ffa* ffa, const lk_tuning* tuning);
/* Synchronises the stream; final cells the last LK_BF16 search rescored. */
int lk_ffa_rescored_cells(lk_ffa* ffa, lk_stream_t stream, uint64_t* n_cells);

/* Per-stage timing with CUDA events recorded on the launching stream
 * (no reference counterpart; used by benchmarks). When enabled, every
 * execute/scores/search call records one event pair per kernel stage. */
enum lk_stage_kind {
    LK_STAGE_INTERLEAVE = 0,  /* series packed into (e, v) pairs for the brute fold */
    LK_STAGE_BRUTE_FOLD = 1,
    LK_STAGE_MERGE = 2,
    LK_STAGE_MERGE_SCORE = 3,
    LK_STAGE_COMPACT = 4,
    LK_STAGE_RESCORE = 5, /* LK_BF16 search: exact rescoring of near-threshold cells */
    LK_STAGE_TRANSFORM = 6, /* Fourier FFA: batched real / inverse real transforms */
    LK_STAGE_SCORE = 7      /* standalone boxcar S/N of a fold back in time */
};
typedef struct lk_stage_time {
    int32_t kind;       /* lk_stage_kind */
    int32_t level;      /* FFA level the stage produces (-1 if none) */
    uint32_t launches;  /* kernels launched by the stage */
    float ms;           /* elapsed GPU time of the last call */
    uint64_t bytes;     /* algorithmic bytes moved (reads + writes) */
} lk_stage_time;
int lk_ffa_set_profiling(lk_ffa* ffa, int enable);
/* Synchronises the stream, then reports the stages of the last call. */
int lk_ffa_get_profile(lk_ffa* ffa, lk_stream_t stream, lk_stage_time* out, uint32_t max_out,
                       uint32_t* n_out);
/* Stage timing of the chunks' executors; the profile of the last execute is
 * summed by stage kind over levels and chunks (level -1). */
int lk_sweep_set_profiling(lk_sweep* sw, int enable);
int lk_sweep_get_profile(lk_sweep* sw, lk_stage_time* out, uint32_t max_out, uint32_t* n_out);
/* Stage timing of the Fourier-domain FFA (as lk_ffa_get_profile). */
int lk_fourier_set_profiling(lk_fourier* f, int enable);
int lk_fourier_get_profile(lk_fourier* f, lk_stream_t stream, lk_stage_time* out,
                           uint32_t max_out, uint32_t* n_out);

/* ---- brute fold (replaces BruteFoldCUDA<float>) ------------------------ */
int lk_brute_fold_create(const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                         uint64_t nbins, uint64_t nsamps, double tsamp, double t_ref,
                         int device, lk_brute_fold** out);
void lk_brute_fold_destroy(lk_brute_fold* bf);
/* d_fold: [nsamps/segment_len, nfreqs, 2, nbins] FP32. */
int lk_brute_fold_execute(lk_brute_fold* bf, const float* d_ts_e, const float* d_ts_v,
                          float* d_fold, lk_stream_t stream);

/* ---- boxcar S/N -------------------------------------------------------- */
/* detection::generate_box_width_trials (lib/score.cpp:390-405): writes up to
 * max_out widths and their number to *n_out. */
int lk_box_width_trials(uint64_t nbins, double ducy_max, double wtsp, uint32_t* out,
                        uint32_t max_out, uint32_t* n_out);
/* d_folds [nprofiles, 2, nbins] (E row, V row). mode LK_SCORE_PER_WIDTH
 * writes [nprofiles, nwidths]; LK_SCORE_MAX writes [nprofiles]. */
int lk_snr_boxcar_3d(const float* d_folds, uint64_t nprofiles, uint32_t nbins,
                     const uint32_t* widths, uint32_t nwidths, int mode, float* d_scores,
                     lk_stream_t stream);
/* d_folds [nprofiles, nbins], S/N divided by stdnoise; [nprofiles] max. */
int lk_snr_boxcar_2d_max(const float* d_folds, uint64_t nprofiles, uint32_t nbins,
                         const uint32_t* widths, uint32_t nwidths, float stdnoise,
                         float* d_scores, lk_stream_t stream);

/* ---- compaction -------------------------------------------------------- */
/* Device scratch bytes lk_compact_ge needs for n inputs. */
uint64_t lk_compact_scratch_bytes(uint64_t n);
/* Keep d_scores[i] >= thr in increasing i: up to max_out (i, score) pairs;
 * *d_count = number passing. d_scratch: lk_compact_scratch_bytes(n) bytes. */
int lk_compact_ge(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx,
                  float* d_vals, uint64_t max_out, uint64_t* d_count, void* d_scratch,
                  lk_stream_t stream);
/* ---- bounded device-side waits ----------------------------------------- */
/* Check of the bounded mbarrier wait the pipelined kernels use (no reference
 * counterpart; the reference's waits are unbounded). One warp waits up to
 * limit_us (1000 .. 500000) on an mbarrier that one arrival completes
 * (complete != 0) or that nothing completes (complete == 0); no asynchronous
 * copy is in flight. Synchronises the stream and writes the status word.
 * Returns LK_ERR_DEVICE_TIMEOUT when the wait gave up (bit 0 of *status
 * set), LK_OK when the barrier completed; the context stays usable. */
int lk_wait_check(uint32_t limit_us, int complete, uint32_t* status, lk_stream_t stream);

/* Allocation-free variant of lk_compact_ge; it has no counterpart in the
 * reference. For callers that may not call cudaMalloc or any allocating
 * routine where they compact (a host framework that owns all device memory
 * through its own pool, or a latency-critical loop where an allocation, which
 * can synchronise the device, is not allowed). The scratch is a static device
 * array inside the library (768 KiB per GPU that loads the library, held
 * until exit), so: n must not exceed 2^28 (larger n is rejected with
 * LK_ERR_INVALID_ARG); calls whose work overlaps on the GPU race on that
 * array and must be serialised. The first call on a device looks up the
 * array's device address with that device current; make that first call
 * before any stream capture. The address is cached per device and context:
 * the first call after the device's context was reset (cudaDeviceReset)
 * looks it up again. Same results as lk_compact_ge. */
int lk_compact_ge_noalloc(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx,
                          float* d_vals, uint64_t max_out, uint64_t* d_count,
                          lk_stream_t stream);

/* ---- pruning leaf step (Taylor basis, nparams 2 or 3) ------------------ */
/* Leaves are [n, nparams + 2, 2] doubles: (value, step) of each Taylor
 * parameter from the highest derivative down to velocity, then (d0, 0) and
 * (f0, basis flag), as core::poly_taylor_seed lays them out. Index arrays on
 * the device are uint32 (the reference uses 64-bit SizeType on the host). */
typedef struct lk_prune lk_prune;

/* cands::PruneStats fields of one level. */
typedef struct lk_prune_stats {
    uint64_t level;
    uint64_t seg_idx;
    uint64_t n_branches;
    uint64_t n_leaves;
    uint64_t n_leaves_phy;
    uint64_t n_leaves_surv;
    float threshold;
    float score_min;
    float score_max;
    float pad;
} lk_prune_stats;

/* One pruning search over the final FFA level of the plan (its nsegments
 * segments, bseg_ffa samples each). max_sugg: world-tree capacity;
 * batch_size: parents per batch (the reference's batch semantics, which
 * decide when the threshold rises); branch_max: most child values of one
 * parameter, 0 for EPMultiPass's rule max(ceil(2 * max branching), 32) over
 * the branching pattern of ref_seg 0 (lib/prune.cpp:648-651);
 * conservative: use_conservative_tile. */
int lk_prune_create(const lk_plan* plan, uint64_t max_sugg, uint64_t batch_size,
                    uint64_t branch_max, int conservative, int device, lk_prune** out);
void lk_prune_destroy(lk_prune* pr);
/* Seed from segment ref_seg of d_ffa_fold ([nsegments, ncoords, 2, nbins],
 * the output of lk_ffa_execute) and run up to n_iters levels, level l using
 * thresholds[l - 1] (host array). stats (host) receives one row for the seed
 * and one per level run, *n_stats their number (stops when no leaf
 * survives). Synchronises the stream several times per level. */
int lk_prune_run(lk_prune* pr, const float* d_ffa_fold, uint64_t ref_seg,
                 const float* thresholds, uint64_t n_thresholds, uint64_t n_iters,
                 lk_prune_stats* stats, uint64_t max_stats, uint64_t* n_stats,
                 lk_stream_t stream);
/* Whether lk_prune_run runs the levels of a small tree (at most 16384
 * parents and a bounded number of children per level) in one persistent
 * cooperative launch, the batch replay done on the device (1, the default;
 * LOKI_B200_PRUNE_TAIL=0 in the environment makes 0 the default) or level by
 * level with host round trips (0). Results are identical. */
int lk_prune_set_tail(lk_prune* pr, int enable);
/* n pruning runs at once on one stream, one executor each (created from one
 * plan with the same sizes; distinct handles): run k seeds from ref_segs[k]
 * and its results are those lk_prune_run gives it. Each run's large levels
 * run level by level; then the small trees' tails of all runs share ONE
 * cooperative launch (its blocks split between the runs); then whatever a
 * tail handed back. stats: [n][max_stats] rows, n_stats[k] rows of run k. The
 * reference runs its segments on a thread pool (lib/prune.cpp:839-926). */
int lk_prune_run_many(lk_prune* const* prs, uint64_t n, const float* d_ffa_fold,
                      const uint64_t* ref_segs, const float* thresholds, uint64_t n_thresholds,
                      uint64_t n_iters, lk_prune_stats* stats, uint64_t max_stats, uint64_t* n_stats,
                      lk_stream_t stream);
/* core::generate_bp_poly_taylor (lib/taylor.cpp:1643-1741), the
 * FFAPlan::get_branching_pattern("taylor", ref_seg) of the reference: the
 * average branching factor of each of the nsegments - 1 pruning levels. */
int lk_plan_branching_pattern(const lk_plan* plan, uint64_t ref_seg, int conservative,
                              double* out, uint64_t max_out, uint64_t* n_out);
/* Polynomial basis of a pruning search (the reference's poly_basis):
 * Taylor (PrunePolyTaylorDPFuncts) or Chebyshev (PrunePolyChebyshevDPFuncts,
 * lib/dynamic.cpp:381-450; lib/chebyshev.cpp). */
enum lk_poly_basis { LK_BASIS_TAYLOR = 0, LK_BASIS_CHEBYSHEV = 1 };
/* lk_prune_create with a basis. Chebyshev: seeds converted to the basis,
 * parents re-centred (coord_prev -> coord_cur) in the branch, and
 * conservative = 1 rejected (the reference throws); branch_max 0 applies
 * EPMultiPass's rule to the basis's branching pattern. */
int lk_prune_create_basis(const lk_plan* plan, uint64_t max_sugg, uint64_t batch_size,
                          uint64_t branch_max, int conservative, int poly_basis, int device,
                          lk_prune** out);
/* FFAPlan::get_branching_pattern(basis, ref_seg): generate_bp_poly_taylor or
 * generate_bp_poly_chebyshev (lib/chebyshev.cpp:1796-1890). */
int lk_plan_branching_pattern_basis(const lk_plan* plan, uint64_t ref_seg, int conservative,
                                    int poly_basis, double* out, uint64_t max_out,
                                    uint64_t* n_out);
/* The end of a pruning run (PruneImpl::run, lib/prune.cpp:136-139,
 * ascend_survivors_batched and report_survivors, lib/prune.cpp:228-334):
 * every survivor's fold rebuilt over all segments searched so far and
 * rescored (the run's scores kept as scores_ep), then its leaf reported at
 * the middle of the data (observer-frame Taylor parameters; Chebyshev leaves
 * converted first). Once per lk_prune_run; d_ffa_fold as given to the run. */
int lk_prune_finalize(lk_prune* pr, const float* d_ffa_fold, lk_stream_t stream);
/* scores_ep of the finalized tree, logical order (max_out >= tree size). */
int lk_prune_get_scores_ep(const lk_prune* pr, float* d_scores_ep, uint64_t max_out,
                           lk_stream_t stream);

/* Surviving leaves after lk_prune_run, in the world tree's logical order.
 * Any of the device outputs may be NULL. */
int lk_prune_tree_size(const lk_prune* pr, uint64_t* n);
int lk_prune_get_tree(const lk_prune* pr, double* d_leaves, float* d_folds, float* d_scores,
                      uint64_t max_out, lk_stream_t stream);

/* Single steps, for callers composing their own level loop. */
/* Seed leaves of the plan's final level, [ncoords, nparams + 2, 2]. */
int lk_taylor_seed(const lk_plan* plan, double* d_leaves, lk_stream_t stream);
/* Branch n parents with dt = scale of the current coordinate. Children are
 * written in parent order (origins: parent index); *n_out (host) = children;
 * nothing is written beyond max_out. Synchronises the stream. */
int lk_taylor_branch(const lk_plan* plan, const double* d_leaves, uint64_t n, double scale_cur,
                     uint64_t branch_max, double* d_out, uint32_t* d_origins, uint64_t max_out,
                     uint64_t* n_out, lk_stream_t stream);
/* coords = {t_add, scale_add, t_cur, scale_cur, t_init, scale_init} (host). */
int lk_taylor_resolve(const lk_plan* plan, const double* d_leaves, uint64_t n,
                      const double* coords, uint32_t* d_param_idx, float* d_phase_shift,
                      lk_stream_t stream);
/* In place on the leaves named by d_indices[0..n) of d_leaves[0..n_leaves);
 * an index at or beyond n_leaves is rejected (LK_ERR_INVALID_ARG, after the
 * other leaves are done). Synchronises the stream. */
int lk_taylor_transform(const lk_plan* plan, double* d_leaves, uint64_t n_leaves,
                        const uint32_t* d_indices, uint64_t n, double t_next, double t_cur,
                        int conservative, lk_stream_t stream);
/* Chebyshev-basis steps (lib/chebyshev.cpp). Leaves keep the Taylor layout:
 * rows 0 .. nparams-1 the coefficients alpha_nparams .. alpha_1, row nparams
 * alpha_0, row nparams + 1 f0, each (value, error). */
/* poly_taylor_to_cheby_batch (ts = scale of coord_init) and
 * poly_cheby_to_taylor_batch (ts = scale of coord_report), in place. */
int lk_taylor_to_cheby(double* d_leaves, uint64_t n, uint32_t nparams, double ts,
                       lk_stream_t stream);
int lk_cheby_to_taylor(double* d_leaves, uint64_t n, uint32_t nparams, double ts,
                       lk_stream_t stream);
/* poly_chebyshev_branch_batch: d_leaves (n parents) are re-centred in place
 * from (t_prev, s_prev) to (t_cur, s_cur), then branched as lk_taylor_branch
 * with the Chebyshev steps. Synchronises the stream. */
int lk_cheby_branch(const lk_plan* plan, double* d_leaves, uint64_t n, double t_cur, double s_cur,
                    double t_prev, double s_prev, uint64_t branch_max, double* d_out,
                    uint32_t* d_origins, uint64_t max_out, uint64_t* n_out, lk_stream_t stream);
/* poly_chebyshev_resolve_batch; coords as for lk_taylor_resolve. */
int lk_cheby_resolve(const lk_plan* plan, const double* d_leaves, uint64_t n,
                     const double* coords, uint32_t* d_param_idx, float* d_phase_shift,
                     lk_stream_t stream);
/* poly_chebyshev_transform_batch from (t_cur, s_cur) to (t_next, s_next),
 * in place on the leaves named by d_indices (checked as lk_taylor_transform).
 * Synchronises the stream. */
int lk_cheby_transform(const lk_plan* plan, double* d_leaves, uint64_t n_leaves,
                       const uint32_t* d_indices, uint64_t n, double t_next, double s_next,
                       double t_cur, double s_cur, lk_stream_t stream);
/* out[i] = folds_tree[indices_tree[i] + physical_start, wrapped once at
 *          capacity] + rotate_right(folds_ffa[indices_ffa[i]], round(phase_shift[i])).
 * n_ffa: rows in d_folds_ffa. A tree index still >= capacity after the wrap
 * or an FFA row >= n_ffa is rejected (LK_ERR_INVALID_ARG) and its output
 * left unwritten. Synchronises the stream. */
int lk_shift_add_batch(const float* d_folds_tree, const uint32_t* d_indices_tree,
                       const float* d_folds_ffa, uint64_t n_ffa, const uint32_t* d_indices_ffa,
                       const float* d_phase_shift, float* d_folds_out, uint32_t nbins,
                       uint64_t n, uint64_t physical_start, uint64_t capacity,
                       lk_stream_t stream);
/* Max-width S/N of [n, 2, nbins] folds into d_scores; indices (input order)
 * with score >= threshold into d_indices, their number into *d_count. */
int lk_score_filter(const float* d_folds, uint64_t n, uint32_t nbins, const uint32_t* widths,
                    uint32_t nwidths, float threshold, float* d_scores, uint32_t* d_indices,
                    uint64_t* d_count, lk_stream_t stream);

/* ---- Monte-Carlo threshold stage ------------------------------------------ */
/* simulate_score_prune_fused of the reference's DynamicThresholdScheme
 * (lib/thresholds.cpp:358-431) with detection::snr_boxcar_threshold_with_cache
 * (lib/score.cpp:434-462), one launch sequence per stage:
 *   out_i = (in[src_i] + noise[row_i]) + signal * signal_scale   (FP32, this order)
 *   kept  = max over widths of S/N_w / sqrt(var_in + var_add) > threshold
 * where row_i = rowmap[i] (NULL: i) selects the noise row and, when
 * signal_per_trial, the signal row ([nbins] shared otherwise); src NULL
 * means src_i = i. Kept trials' folds are written to d_folds_out in trial
 * order, their noise rows to d_ids_out (may be NULL), their number to
 * *d_count; d_counts[k] = trials whose maximum S/N > thresholds[k] (host
 * array of n_thr <= 64 entries); with d_class (one byte per noise row, may
 * be NULL) d_counts[n_thr + k] counts the same among trials whose row is
 * flagged (e.g. the ones carrying a signal, for detection probabilities).
 * d_max_snr (may be NULL) receives every trial's maximum S/N. The noise is
 * the caller's (drawn on the host, so the CPU reference can use the same
 * numbers). */
typedef struct lk_mc lk_mc;
int lk_mc_create(uint64_t max_trials, uint32_t nbins, const uint32_t* widths, uint32_t nwidths,
                 int device, lk_mc** out);
void lk_mc_destroy(lk_mc* mc);
/* ntrials_in: rows of d_folds_in; nrows: rows of d_noise (and of d_signal
 * when signal_per_trial). A src or rowmap entry outside them is read as row
 * 0 and flagged; lk_mc_status reports (and clears) the flag. */
int lk_mc_stage(lk_mc* mc, const float* d_folds_in, uint64_t ntrials_in, const uint32_t* d_src,
                uint64_t ntrials, const float* d_noise, uint64_t nrows, const float* d_signal,
                int signal_per_trial,
                float signal_scale, const uint32_t* d_rowmap, float var_in, float var_add,
                float threshold, const float* thresholds, uint32_t n_thr,
                const uint8_t* d_class, float* d_folds_out, uint32_t* d_ids_out,
                uint64_t* d_count, uint64_t* d_counts, float* d_max_snr, lk_stream_t stream);
/* Synchronises the stream; *status = non-zero when an index was out of range
 * since the last call (and clears it). */
int lk_mc_status(lk_mc* mc, lk_stream_t stream, uint32_t* status);

/* ---- DynamicThresholdScheme beam search ---------------------------------- */
/* Replaces detection::DynamicThresholdScheme / DynamicThresholdSchemeCUDA
 * (include/loki/detection/thresholds.hpp:65-164, lib/thresholds.cpp:560-907,
 * lib/thresholds_cuda.cu): for every stage and every threshold of the
 * stage's beam, every neighbouring previous state is advanced by simulating
 * ntrials H0 and H1 folds, scoring them and keeping the survivors; each
 * (threshold, probability bin) cell keeps the first transition with the
 * smallest cumulative complexity. Noise comes from a counter-based generator
 * (Philox4x32-10 words through the reference's normal quantile table), so a
 * run is reproducible from `seed`. */
typedef struct lk_dts lk_dts;
/* detection::State (include/loki/detection/thresholds.hpp:17-29), same fields
 * and order; is_empty is 1 for a cell no transition reached. */
typedef struct lk_dts_state {
    float success_h0;
    float success_h1;
    float complexity;
    float complexity_cumul;
    float success_h1_cumul;
    float nbranches;
    float threshold;
    float cost;
    float threshold_prev;
    float success_h1_cumul_prev;
    uint8_t is_empty;
    uint8_t pad[3];
} lk_dts_state;
/* The reference constructor's arguments (defaults there: nbins 64, ntrials
 * 1024, nprobs 10, prob_min 0.05, snr_final 8, nthresholds 100, ducy_max 0.3,
 * wtsp 1, beam_width 0.7, trials_start 1) plus the generator seed. */
typedef struct lk_dts_config {
    const float* branching_pattern; /* host, nstages entries */
    uint32_t nstages;
    float ref_ducy;
    uint32_t nbins;
    uint32_t ntrials;
    uint32_t nprobs;
    float prob_min;
    float snr_final;
    uint32_t nthresholds;
    float ducy_max;
    float wtsp;
    float beam_width;
    uint32_t trials_start;
    uint64_t seed;
} lk_dts_config;
int lk_dts_create(const lk_dts_config* cfg, int device, lk_dts** out);
void lk_dts_destroy(lk_dts* dts);
/* DynamicThresholdScheme::run(thres_neigh): the whole scheme on `stream`;
 * synchronises it and keeps the states on the host. */
int lk_dts_run(lk_dts* dts, uint32_t thres_neigh, lk_stream_t stream);
int lk_dts_info(const lk_dts* dts, uint32_t* nstages, uint32_t* nthresholds, uint32_t* nprobs,
                uint32_t* nbins, uint32_t* nwidths);
/* Host arrays (NULL skips one): profile [nbins], thresholds [nthresholds],
 * probs [nprobs], guess path [nstages], box widths [nwidths]. */
int lk_dts_arrays(const lk_dts* dts, float* profile, float* thresholds, float* probs,
                  float* guess_path, uint32_t* widths);
/* Transitions the last lk_dts_run simulated (each: ntrials H0 and ntrials
 * H1 folds built and scored). */
int lk_dts_transitions(const lk_dts* dts, uint64_t* n);
/* get_states: [nstages][nthresholds][nprobs] after lk_dts_run; n = capacity. */
int lk_dts_states(const lk_dts* dts, lk_dts_state* out, uint64_t n);
/* get_best_path_thresholds(min_pd): *n thresholds (0 when no final state
 * reaches min_pd); out holds nstages entries. */
int lk_dts_best_path(const lk_dts* dts, float min_pd, float* out, uint32_t* n);
/* Host-only set-up (no device): the arrays lk_dts_arrays reports for cfg
 * (each output may be NULL; widths holds up to 32 entries, *nwidths set). */
int lk_dts_plan(const lk_dts_config* cfg, float* profile, float* thresholds, float* probs,
                float* guess_path, uint32_t* widths, uint32_t* nwidths);
/* The normal quantile table of the generator (n >= 131073 entries). */
int lk_dts_normal_lut(float* out, uint64_t n);

#ifdef __cplusplus
}
#endif

#endif /* LOKI_B200_H */
