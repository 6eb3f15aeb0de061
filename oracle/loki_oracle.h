/* Test infrastructure only: the CPU oracle for the loki time-domain FFA path.
 *
 * A plain-C restatement of the reference's algorithm, used by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg as the checker.
 * The product (loki_b200) never links or calls it. Every function names the
 * reference file:line it restates. Arithmetic is written operation by
 * operation in the reference's order so that, built with
 * -O2 -fno-fast-math -ffp-contract=off, the results are bit-identical to the
 * reference's own code built with the same flags (checked against
 * oracle/_ref in tests/test_oracle_vs_ref.py and the committed fixtures).
 */
#ifndef LOKI_ORACLE_H
#define LOKI_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LKO_MAX_LEVELS 40
#define LKO_MAX_PARAMS 5
#define LKO_MAX_WIDTHS 64

/* Search configuration (subset of PulsarSearchConfig, include/loki/search/
 * configs.hpp:25-47). limits holds (min, max) pairs ordered (..., accel, freq).
 * bseg_brute / bseg_ffa == 0 select the reference defaults. */
typedef struct lko_cfg {
    uint64_t nsamps;
    double tsamp;
    uint64_t nbins;
    double eta;
    uint32_t nparams;
    double limits[2 * LKO_MAX_PARAMS];
    uint64_t bseg_brute;
    uint64_t bseg_ffa;
    double ducy_max;
    double wtsp;
} lko_cfg;

/* FFAPlanBase geometry (lib/plans.cpp:264-320). */
typedef struct lko_plan {
    uint32_t nparams;
    uint32_t n_levels;
    uint64_t nsamps;
    uint64_t nbins;
    double tsamp;
    double eta;
    double tseg_brute;
    uint64_t bseg_brute;
    uint64_t bseg_ffa;
    double limits[2 * LKO_MAX_PARAMS];
    uint64_t segment_lens[LKO_MAX_LEVELS];
    uint64_t nsegments[LKO_MAX_LEVELS];
    double tsegments[LKO_MAX_LEVELS];
    uint64_t ncoords[LKO_MAX_LEVELS];
    uint32_t ncoords_offsets[LKO_MAX_LEVELS + 1];
    uint64_t param_counts[LKO_MAX_LEVELS][LKO_MAX_PARAMS];
    double dparams[LKO_MAX_LEVELS][LKO_MAX_PARAMS];
    uint64_t buffer_size;     /* max over levels of nseg*ncoords*2*nbins */
    uint64_t coord_size;      /* sum over levels of ncoords */
    uint32_t n_widths;        /* generate_box_width_trials(nbins, ...) */
    uint64_t widths[LKO_MAX_WIDTHS];
} lko_plan;

/* FFACoordFreq / FFACoord (include/loki/common/coord.hpp:15-25). */
typedef struct lko_coord_freq {
    uint32_t idx;
    float shift;
} lko_coord_freq;

typedef struct lko_coord {
    uint32_t i_tail;
    float shift_tail;
    uint32_t i_head;
    float shift_head;
} lko_coord;

const char* lko_last_error(void);

/* Plan construction: 0 on success, non-zero with lko_last_error() set. */
int lko_plan_create(const lko_cfg* cfg, lko_plan* out);

/* Scalar phase / grid helpers (lib/loki/psr_utils.hpp:32-63, 235-320). */
float lko_phase_idx(double proper_time, double freq, uint64_t nbins, double delay);
uint32_t lko_phase_idx_uint(double proper_time, double freq, uint64_t nbins, double delay);
double lko_param_val_at_idx(double vmin, double vmax, uint64_t count, uint64_t i);
uint64_t lko_nearest_idx(double val, double vmin, double vmax, uint64_t count);
uint64_t lko_range_param_count(double vmin, double vmax, double dv);
/* psr_utils::range_param (lib/loki/psr_utils.hpp:254-270); returns npoints. */
uint64_t lko_range_param(double vmin, double vmax, double dv, double* out, uint64_t max_out);
uint64_t lko_box_widths(uint64_t nbins, double ducy_max, double wtsp, uint64_t* out,
                        uint64_t max_out);

/* Coordinate tables of every level, flat, coord_size entries (level 0 left
 * zero as in the reference). */
int lko_resolve_freq(const lko_plan* plan, lko_coord_freq* out);
int lko_resolve_taylor(const lko_plan* plan, lko_coord* out);

/* Brute fold (lib/fold.cpp:113-142, lib/kernels.cpp:550-580,1132-1154).
 * out: [nsamps/segment_len, nfreqs, 2, nbins]. */
int lko_brute_fold(const float* ts_e, const float* ts_v, uint64_t nsamps,
                   const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                   uint64_t nbins, double tsamp, double t_ref, float* out);

/* Phase map of the brute fold, uint32 [nfreqs, segment_len]. */
void lko_phase_map(const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                   uint64_t nbins, double tsamp, double t_ref, uint32_t* out);

/* One merge level (lib/kernels.cpp:118-146,722-827 and 71-112,829-940). */
void lko_merge_freq(const float* fold_in, float* fold_out, const lko_coord_freq* coords,
                    uint64_t ncoords_cur, uint64_t ncoords_prev, uint64_t nsegments,
                    uint64_t nbins);
void lko_merge_taylor(const float* fold_in, float* fold_out, const lko_coord* coords,
                      uint64_t ncoords_cur, uint64_t ncoords_prev, uint64_t nsegments,
                      uint64_t nbins);

/* Whole FFA (lib/ffa.cpp:242-310). level_out selects the level whose fold is
 * written to fold_out (n_levels-1 for the final fold). */
int lko_ffa(const lko_plan* plan, const float* ts_e, const float* ts_v,
            uint32_t level_out, float* fold_out);

/* Boxcar S/N (lib/score.cpp:95-172, lib/utils.cpp:22-67). */
void lko_snr_boxcar_3d(const float* folds, uint64_t nprofiles, uint64_t nbins,
                       const uint64_t* widths, uint64_t nwidths, float* scores);
void lko_snr_boxcar_3d_max(const float* folds, uint64_t nprofiles, uint64_t nbins,
                           const uint64_t* widths, uint64_t nwidths, float* scores);
void lko_snr_boxcar_2d_max(const float* folds, uint64_t nprofiles, uint64_t nbins,
                           const uint64_t* widths, uint64_t nwidths, float stdnoise,
                           float* scores);
void lko_circular_prefix_sum(const float* x, float* out, uint64_t nbins, uint64_t nsum);

/* Threshold compaction `score >= snr_min` in flat order
 * (lib/ffa_freq_sweep.cpp:182-195). Returns the number kept. */
/* FP64 FFA + boxcar S/N of every final cell and width, [ncoords, nw]
 * doubles (same phase map, coordinates and shifts as the FP32 path). */
int lko_ffa_scores64(const lko_plan* plan, const float* ts_e, const float* ts_v,
                     const uint64_t* widths, uint64_t nw, double* scores);

uint64_t lko_compact(const float* scores, uint64_t n, float snr_min, uint32_t* idx_out,
                     float* score_out);

/* ---- pruning leaf step (Taylor basis, nparams 2 or 3) ---------------------- */

/* psr_utils::MiddleOutScheme (lib/loki/psr_utils.hpp:327-502) at one level:
 * out[0] = segment index, out[1..2] = get_coord, out[3..4] =
 * get_current_coord, out[5..6] = get_segment_coord. */
int lko_middle_out(uint64_t nsegments, uint64_t ref_idx, double tsegment, uint64_t level,
                   double* out);

/* core::poly_taylor_seed (lib/taylor.cpp:1197-1257) over the final level of
 * the plan: leaves [ncoords, nparams + 2, 2]. Returns the number of leaves
 * (0 with lko_last_error() set on failure). */
uint64_t lko_taylor_seed(const lko_plan* plan, double* leaves_out);

/* poly_taylor_branch_{accel,jerk}_batch (lib/taylor.cpp:24-314). Children
 * counts are computed first: *n_out receives the number of children, and
 * nothing is written when it exceeds cap_out (returns 2). Returns 1 with the
 * reference's message when a parameter needs more than branch_max points. */
int lko_taylor_branch(const double* leaves, uint64_t n, uint32_t nparams, double t_cur,
                      double scale_cur, uint64_t nbins, double eta, uint64_t branch_max,
                      double* leaves_out, uint64_t* origins_out, uint64_t cap_out,
                      uint64_t* n_out);

/* poly_taylor_resolve_{accel,jerk}_batch (lib/taylor.cpp:492-619) against the
 * final level of the plan. coords = {t_add, s_add, t_cur, s_cur, t_init,
 * s_init}. */
void lko_taylor_resolve(const lko_plan* plan, const double* leaves, uint64_t n,
                        const double* coords, uint64_t* param_idx, float* phase_shift);

/* poly_taylor_transform_{accel,jerk}_batch<Conservative> (lib/taylor.cpp:
 * 881-1005), in place on the leaves named by indices. */
void lko_taylor_transform(double* leaves, const uint64_t* indices, uint64_t n, uint32_t nparams,
                          double t_next, double t_cur, int conservative);

/* kernels::shift_add_linear_batch (lib/kernels.cpp:1328-1355). */
void lko_shift_add_batch(const float* folds_tree, const uint64_t* indices_tree,
                         const float* folds_ffa, const uint64_t* indices_ffa,
                         const float* phase_shift, float* folds_out, uint64_t nbins,
                         uint64_t n_leaves, uint64_t physical_start_idx, uint64_t capacity);

/* detection::score_and_filter_max_with_cache (lib/score.cpp:213-259):
 * returns the number of indices (input order) with score >= threshold. */
uint64_t lko_score_filter(const float* folds, uint64_t n, uint64_t nbins,
                          const uint64_t* widths, uint64_t nwidths, float threshold,
                          float* scores, uint64_t* indices);

/* cands::PruneStats fields of one level. */
typedef struct lko_prune_stats {
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
} lko_prune_stats;

/* One pruning run (lib/prune.cpp:181-226 initialize, :429-620 levels) with
 * the WorldTree circular buffer (lib/world_tree.cpp:237-276,361-422,
 * 557-669). ffa_fold is the final FFA level [nsegments, ncoords, 2, nbins];
 * thresholds[level - 1] is the level's threshold. stats receives n_iters + 1
 * rows at most; the final tree (logical order) is copied out when it fits
 * cap_out. */
/* Chebyshev basis of the pruning leaf step (lib/chebyshev.cpp). Leaves keep
 * the Taylor layout; co for resolve = {t_add, s_add, t_cur, s_cur, t_init,
 * s_init}. lko_cheby_branch transforms `leaves` in place (coord_prev ->
 * coord_cur) before branching, as the reference does. */
void lko_taylor_to_cheby(double* leaves, uint64_t n, uint32_t nparams, double ts);
void lko_cheby_to_taylor(double* leaves, uint64_t n, uint32_t nparams, double ts);
void lko_cheby_transform(double* leaves, const uint64_t* indices, uint64_t n, uint32_t nparams,
                         double t_next, double s_next, double t_cur, double s_cur);
int lko_cheby_branch(double* leaves, uint64_t n, uint32_t nparams, double t_cur, double s_cur,
                     double t_prev, double s_prev, uint64_t nbins, double eta,
                     uint64_t branch_max, double* out, uint64_t* origins, uint64_t cap_out,
                     uint64_t* n_out);
void lko_cheby_resolve(const lko_plan* plan, const double* leaves, uint64_t n, const double* co,
                       uint64_t* param_idx, float* phase_shift);
int lko_prune_run_basis(const lko_plan* plan, int basis, int conservative, const float* ffa_fold,
                        const float* thresholds, uint64_t n_thresholds, uint64_t ref_seg,
                        uint64_t max_sugg, uint64_t batch_size, uint64_t branch_max,
                        uint64_t n_iters, lko_prune_stats* stats, uint64_t* n_stats,
                        double* leaves_out, float* folds_out, float* scores_out, uint64_t cap_out,
                        uint64_t* n_out);
/* The end of a pruning run (PruneImpl::run, lib/prune.cpp:136-139): the n
 * surviving leaves (logical order, after prune_level levels from ref_seg)
 * ascended to the middle of the data -- folds rebuilt over every segment so
 * far, scores_ep = the scores before, scores = the new folds' scores -- and
 * the leaves reported there. */
int lko_prune_finalize(const lko_plan* plan, int basis, const float* ffa_fold, uint64_t ref_seg,
                       uint64_t prune_level, double* leaves, float* folds, float* scores,
                       float* scores_ep, uint64_t n);
int lko_prune_run(const lko_plan* plan, int conservative, const float* ffa_fold,
                  const float* thresholds, uint64_t n_thresholds, uint64_t ref_seg,
                  uint64_t max_sugg, uint64_t batch_size, uint64_t branch_max, uint64_t n_iters,
                  lko_prune_stats* stats, uint64_t* n_stats, double* leaves_out,
                  float* folds_out, float* scores_out, uint64_t cap_out, uint64_t* n_out);

/* ---- Monte-Carlo threshold stage ------------------------------------------ */

/* Largest boxcar S/N of one 2-D profile with every width's S/N divided by
 * stdnoise (detection::snr_boxcar_threshold_with_cache, lib/score.cpp:434-462,
 * decides S/N > threshold for some width, i.e. this maximum > threshold). */
float lko_snr_max_div(const float* prof, uint64_t nbins, const uint64_t* widths, uint64_t nw,
                      float stdnoise);

/* One fused stage of simulate_score_prune_fused (lib/thresholds.cpp:358-431);
 * see loki_oracle.c for the argument meanings. Returns the trials kept. */
uint64_t lko_mc_stage(const float* folds_in, const uint32_t* src, uint64_t ntrials,
                      uint64_t nbins, const float* noise, const float* signal,
                      int signal_per_trial, float signal_scale, const uint32_t* rowmap,
                      float var_in, float var_add, const uint64_t* widths, uint64_t nw,
                      float threshold, const float* thr, uint64_t n_thr, const uint8_t* cls,
                      float* folds_out, uint32_t* ids_out, uint64_t* counts, float* max_snr);

/* ---- DynamicThresholdScheme beam search (lib/thresholds.cpp:560-907) ---- */
typedef struct lko_dts_state {
    float success_h0, success_h1, complexity, complexity_cumul, success_h1_cumul, nbranches,
        threshold, cost, threshold_prev, success_h1_cumul_prev;
    uint8_t is_empty;
    uint8_t pad[3];
} lko_dts_state;
typedef struct lko_dts_config {
    const float* branching_pattern;
    uint32_t nstages;
    float ref_ducy;
    uint32_t nbins, ntrials, nprobs;
    float prob_min, snr_final;
    uint32_t nthresholds;
    float ducy_max, wtsp, beam_width;
    uint32_t trials_start;
    uint64_t seed;
} lko_dts_config;
double lko_normal_quantile(double p);
void lko_dts_normal_lut(float* out);
void lko_dts_thresholds(float snr_start, float snr_final, uint32_t n, float* out);
void lko_dts_probs(uint32_t n, float prob_min, float* out);
void lko_dts_profile(uint32_t nbins, float ducy, float center, float* out);
void lko_dts_guess(uint32_t nstages, float snr_bound, const float* branching, uint32_t trials_start,
                   float min_trials, float* out);
uint32_t lko_dts_neighbours(const uint32_t* idx, uint32_t n, uint32_t target, uint32_t num,
                            uint32_t* out);
int64_t lko_dts_lower_bin(const float* range, uint32_t n, float v);
lko_dts_state lko_dts_gen_next(const lko_dts_state* s, float threshold, float s0, float s1,
                               float nbranches);
void lko_philox4x32_10(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]);
float lko_dts_normal(uint32_t r, const float* lut);
uint32_t lko_dts_resample(uint32_t range, uint32_t i, uint32_t tid2, uint32_t stage_code,
                          uint32_t k0, uint32_t k1);
/* The scheme's first stages_run stages (0: all); states [nstages][nthresholds][nprobs]
 * (stages not run stay empty). */
int lko_dts_run(const lko_dts_config* cfg, uint32_t thres_neigh, uint32_t stages_run,
                lko_dts_state* states);

/* Fourier-domain FFA in double (FFA<ComplexType>). Complex arrays are
 * interleaved (re, im) doubles; folds [nseg][ncoords][2][nbins/2 + 1]. */
int lko_fourier_brute_fold(const float* ts_e, const float* ts_v, uint64_t nsamps,
                           const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                           uint64_t nbins, double tsamp, double t_ref, double* out);
void lko_fourier_merge(const double* in, double* out, const void* coords, int taylor,
                       uint64_t ncur, uint64_t nprev, uint64_t nseg, uint64_t nbins);
void lko_irfft(const double* in, double* out, uint64_t nprof, uint64_t n);
void lko_rfft(const double* in, double* out, uint64_t nprof, uint64_t n);
int lko_ffa_fourier(const lko_plan* p, const float* ts_e, const float* ts_v, uint32_t level_out,
                    uint64_t nbins_min_lossy, double* fold_out);
int lko_ffa_fourier_scores64(const lko_plan* p, const float* ts_e, const float* ts_v,
                             uint64_t nbins_min_lossy, const uint64_t* widths, uint64_t nw,
                             double* scores);

#ifdef __cplusplus
}
#endif

#endif /* LOKI_ORACLE_H */
