// Test infrastructure only: a C-ABI over the reference's own CPU code.
//
// This file is compiled together with the UNMODIFIED reference sources (read
// in place from the reference checkout by oracle/Makefile) into
// oracle/_ref/libloki_ref_*.so. It is never part of the product: only tests,
// the golden-fixture generator and bench.py's reference arm load it, as the
// checker and as the timed CPU baseline.
//
// Each entry point wraps one reference call and converts C++ exceptions into
// a non-zero return code plus a message readable with lkref_last_error().
//
//   lkref_ffa_*           -> algorithms::FFA<float> (lib/ffa.cpp:26-361)
//   lkref_resolve_*       -> plans::FFAPlanBase::resolve_coordinates[_freq]
//                            (lib/plans.cpp:64-132)
//   lkref_brute_fold      -> algorithms::compute_brute_fold<float>
//                            (lib/fold.cpp:176-190)
//   lkref_snr_boxcar_3d*  -> detection::snr_boxcar_3d[_max] (lib/score.cpp:498-529)
//   lkref_box_widths      -> detection::generate_box_width_trials
//                            (lib/score.cpp:390-405)
//   lkref_phase_idx*      -> psr_utils::get_phase_idx[_uint]
//                            (lib/loki/psr_utils.hpp:32-63)
//   lkref_middle_out      -> psr_utils::MiddleOutScheme (lib/loki/psr_utils.hpp:327-502)
//   lkref_taylor_*        -> core::poly_taylor_{seed,branch,resolve,transform}_batch
//                            (lib/taylor.cpp:24-314,492-619,881-1005,1197-1257)
//   lkref_shift_add_batch -> kernels::shift_add_linear_batch (lib/kernels.cpp:1328-1355)
//   lkref_score_filter    -> detection::score_and_filter_max_with_cache
//                            (lib/score.cpp:213-259)
//   lkref_branch_max      -> EPMultiPass's branch_max rule (lib/prune.cpp:648-651)
//   lkref_snr_threshold   -> detection::snr_boxcar_threshold_with_cache
//                            (lib/score.cpp:434-462)
//   lkref_dts_*           -> the DynamicThresholdScheme set-up and pieces
//                            (detail::compute_thresholds / compute_probs /
//                            bound_scheme / get_best_path_thresholds,
//                            lib/scheme.cpp; generate_folded_profile,
//                            lib/simulation.cpp:12-50; find_neighbouring_indices
//                            / find_lower_bin_index, lib/utils.cpp:138-185;
//                            State::gen_next, thresholds.hpp:32-58) and
//                            lkref_dts_run, the scheme's stage loop
//                            (lib/thresholds.cpp:748-907) restated over those
//                            pieces and snr_boxcar_threshold_with_cache,
//                            because thresholds.cpp itself needs HDF5; its
//                            noise is the counter-based stream of the oracle
//                            (Philox words through the normal quantile table)
//   lkref_prune_run       -> PruneImpl::initialize + execute_iteration[_batched]
//                            (lib/prune.cpp:181-226,429-620), restated here
//                            because prune.cpp itself needs HDF5 and a
//                            thread pool; every step calls the reference's
//                            own PruneDPFuncts (lib/dynamic.cpp) and
//                            WorldTree (lib/world_tree.cpp).

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <optional>
#include <span>
#include <string>
#include <vector>

#include <omp.h>
#include <spdlog/spdlog.h>

#include "loki/algorithms/ffa.hpp"
#include "loki/algorithms/fold.hpp"
#include "loki/algorithms/regions.hpp"
#include "loki/common/coord.hpp"
#include "loki/common/plans.hpp"
#include "loki/common/types.hpp"
#include "loki/core/dynamic.hpp"
#include "loki/core/chebyshev.hpp"
#include "loki/core/taylor.hpp"
#include "loki/detection/score.hpp"
#include "loki/detection/thresholds.hpp"
#include "loki/scheme.hpp"
#include "loki/simulation/simulation.hpp"
#include "loki/utils.hpp"
#include "loki/kernels.hpp"
#include "loki/psr_utils.hpp"
#include "loki/search/configs.hpp"
#include "loki/utils/workspace.hpp"
#include "loki/utils/world_tree.hpp"

namespace {

thread_local std::string g_last_error;

template <class F> int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
    } catch (...) {
        g_last_error = "unknown C++ exception";
    }
    return 1;
}

struct QuietLogs {
    QuietLogs() { spdlog::set_level(spdlog::level::warn); }
};
const QuietLogs g_quiet_logs;

} // namespace

extern "C" {

// Search configuration in plain C types. `limits` holds nparams (min, max)
// pairs in the reference order (..., accel, freq). bseg_brute / bseg_ffa of 0
// select the reference defaults (lib/configs.cpp:295-302).
struct lkref_cfg {
    uint64_t nsamps;
    double tsamp;
    uint64_t nbins;
    double eta;
    uint32_t nparams;
    double limits[10];
    uint64_t bseg_brute;
    uint64_t bseg_ffa;
    int32_t nthreads;
    double ducy_max;
    double wtsp;
};

struct lkref_ffa {
    std::unique_ptr<loki::search::PulsarSearchConfig> cfg;
    std::unique_ptr<loki::algorithms::FFA<float>> ffa;
};

const char* lkref_last_error(void) { return g_last_error.c_str(); }

int lkref_max_threads(void) { return omp_get_max_threads(); }

static loki::search::PulsarSearchConfig make_cfg(const lkref_cfg* c, bool use_fourier = false) {
    std::vector<loki::ParamLimit> lims(c->nparams);
    for (uint32_t i = 0; i < c->nparams; ++i) {
        lims[i] = {.min = c->limits[2 * i], .max = c->limits[(2 * i) + 1]};
    }
    std::optional<loki::SizeType> bb;
    std::optional<loki::SizeType> bf;
    if (c->bseg_brute != 0) {
        bb = c->bseg_brute;
    }
    if (c->bseg_ffa != 0) {
        bf = c->bseg_ffa;
    }
    return {c->nsamps, c->tsamp, c->nbins, c->eta, lims, c->ducy_max, c->wtsp,
            use_fourier, c->nthreads,
            /*max_process_memory_gb=*/8.0, /*octave_scale=*/2.0,
            /*nbins_max=*/1024, /*nbins_min_lossy_bf=*/64, bb, bf};
}

int lkref_ffa_create(const lkref_cfg* c, lkref_ffa** out) {
    return guarded([&] {
        auto h  = std::make_unique<lkref_ffa>();
        h->cfg  = std::make_unique<loki::search::PulsarSearchConfig>(make_cfg(c));
        h->ffa  = std::make_unique<loki::algorithms::FFA<float>>(*h->cfg, false);
        *out    = h.release();
    });
}

void lkref_ffa_destroy(lkref_ffa* h) { delete h; }

// Plan geometry. Arrays must hold at least n_levels (+1 for offsets) entries;
// counts holds n_levels * nparams entries.
int lkref_ffa_info(const lkref_ffa* h,
                   uint64_t* n_levels,
                   uint64_t* buffer_size,
                   uint64_t* fold_size,
                   uint64_t* brute_fold_size,
                   uint64_t* coord_size,
                   uint64_t* bseg_brute,
                   uint64_t max_levels,
                   uint64_t* segment_lens,
                   uint64_t* nsegments,
                   uint64_t* ncoords,
                   uint32_t* ncoords_offsets,
                   uint64_t* counts,
                   double* dparams) {
    return guarded([&] {
        const auto& plan = h->ffa->get_plan();
        const auto L     = plan.get_n_levels();
        const auto np    = plan.get_n_params();
        *n_levels        = L;
        *buffer_size     = plan.get_buffer_size();
        *fold_size       = plan.get_fold_size();
        *brute_fold_size = plan.get_brute_fold_size();
        *coord_size      = plan.get_coord_size();
        *bseg_brute      = h->cfg->get_bseg_brute();
        if (L > max_levels) {
            throw std::runtime_error("lkref_ffa_info: max_levels too small");
        }
        for (loki::SizeType l = 0; l < L; ++l) {
            segment_lens[l] = plan.get_segment_lens()[l];
            nsegments[l]    = plan.get_nsegments()[l];
            ncoords[l]      = plan.get_ncoords()[l];
            for (loki::SizeType p = 0; p < np; ++p) {
                counts[(l * np) + p]  = plan.get_param_counts()[l][p];
                dparams[(l * np) + p] = plan.get_dparams()[l][p];
            }
        }
        for (loki::SizeType l = 0; l <= L; ++l) {
            ncoords_offsets[l] = plan.get_ncoords_offsets()[l];
        }
    });
}

// fold must hold buffer_size floats; on return its first fold_size floats are
// the final-level fold [nseg, counts..., 2, nbins].
int lkref_ffa_execute(lkref_ffa* h,
                      const float* ts_e,
                      const float* ts_v,
                      uint64_t nsamps,
                      float* fold,
                      uint64_t fold_len) {
    return guarded([&] {
        h->ffa->execute(std::span<const float>(ts_e, nsamps),
                        std::span<const float>(ts_v, nsamps),
                        std::span<float>(fold, fold_len));
    });
}

// ---- Fourier-domain FFA (FFA<ComplexType>, lib/ffa.cpp) ----------------
struct lkref_fourier {
    std::unique_ptr<loki::search::PulsarSearchConfig> cfg;
    std::unique_ptr<loki::algorithms::FFA<loki::ComplexType>> ffa;
};

int lkref_fourier_create(const lkref_cfg* c, lkref_fourier** out) {
    return guarded([&] {
        auto h = std::make_unique<lkref_fourier>();
        h->cfg = std::make_unique<loki::search::PulsarSearchConfig>(make_cfg(c, true));
        h->ffa = std::make_unique<loki::algorithms::FFA<loki::ComplexType>>(*h->cfg, false);
        *out   = h.release();
    });
}

void lkref_fourier_destroy(lkref_fourier* h) { delete h; }

// Complex counts: buffer (ping-pong side), final fold; final fold in floats
// once back in time.
int lkref_fourier_info(const lkref_fourier* h, uint64_t* buffer_size, uint64_t* fold_size,
                       uint64_t* fold_size_time) {
    return guarded([&] {
        const auto& plan = h->ffa->get_plan();
        *buffer_size     = plan.get_buffer_size();
        *fold_size       = plan.get_fold_size();
        *fold_size_time  = plan.get_fold_size_time();
    });
}

// FFA<ComplexType>::execute(span<ComplexType>): fold holds buffer_size
// complex values as interleaved floats; its first fold_size are the result.
int lkref_fourier_execute(lkref_fourier* h, const float* ts_e, const float* ts_v, uint64_t nsamps,
                          float* fold, uint64_t fold_len_complex) {
    return guarded([&] {
        h->ffa->execute(std::span<const float>(ts_e, nsamps), std::span<const float>(ts_v, nsamps),
                        std::span<loki::ComplexType>(reinterpret_cast<loki::ComplexType*>(fold),
                                                     fold_len_complex));
    });
}

// FFA<ComplexType>::execute(span<float>): back to time by the inverse real
// transform; fold holds 2 * buffer_size floats, its first fold_size_time the
// result.
int lkref_fourier_execute_time(lkref_fourier* h, const float* ts_e, const float* ts_v,
                               uint64_t nsamps, float* fold, uint64_t fold_len) {
    return guarded([&] {
        h->ffa->execute(std::span<const float>(ts_e, nsamps), std::span<const float>(ts_v, nsamps),
                        std::span<float>(fold, fold_len));
    });
}

// compute_ffa_scores with use_fourier = true (lib/ffa.cpp:444-466).
int lkref_fourier_scores(const lkref_cfg* c, const float* ts_e, const float* ts_v, uint64_t nsamps,
                         float* scores, uint64_t len) {
    return guarded([&] {
        const auto cfg = make_cfg(c, true);
        auto [sc, plan] = loki::algorithms::compute_ffa_scores(
            std::span<const float>(ts_e, nsamps), std::span<const float>(ts_v, nsamps), cfg, true,
            false);
        if (sc.size() != len) {
            throw std::runtime_error("lkref_fourier_scores: output size mismatch");
        }
        std::memcpy(scores, sc.data(), sc.size() * sizeof(float));
    });
}

// compute_brute_fold<ComplexType> (lib/fold.cpp): [nseg, nfreqs, 2, nbins/2+1]
// complex as interleaved floats.
int lkref_brute_fold_complex(const float* ts_e, const float* ts_v, uint64_t nsamps,
                             const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                             uint64_t nbins, double tsamp, double t_ref, int nthreads, float* out,
                             uint64_t out_len_complex) {
    return guarded([&] {
        auto fold = loki::algorithms::compute_brute_fold<loki::ComplexType>(
            std::span<const float>(ts_e, nsamps), std::span<const float>(ts_v, nsamps),
            std::span<const double>(freqs, nfreqs), segment_len, nbins, tsamp, t_ref, nthreads);
        if (fold.size() != out_len_complex) {
            throw std::runtime_error("lkref_brute_fold_complex: output size mismatch");
        }
        std::memcpy(out, fold.data(), fold.size() * sizeof(loki::ComplexType));
    });
}

// Coordinates of every level in one flat array (coord_size entries).
int lkref_resolve_freq(const lkref_cfg* c, void* coords_out, uint64_t n) {
    return guarded([&] {
        auto cfg = make_cfg(c);
        loki::plans::FFAPlan<float> plan(cfg);
        plan.resolve_coordinates_freq(std::span<loki::coord::FFACoordFreq>(
            static_cast<loki::coord::FFACoordFreq*>(coords_out), n));
    });
}

int lkref_resolve(const lkref_cfg* c, void* coords_out, uint64_t n) {
    return guarded([&] {
        auto cfg = make_cfg(c);
        loki::plans::FFAPlan<float> plan(cfg);
        plan.resolve_coordinates(std::span<loki::coord::FFACoord>(
            static_cast<loki::coord::FFACoord*>(coords_out), n));
    });
}

int lkref_brute_fold(const float* ts_e,
                     const float* ts_v,
                     uint64_t nsamps,
                     const double* freqs,
                     uint64_t nfreqs,
                     uint64_t segment_len,
                     uint64_t nbins,
                     double tsamp,
                     double t_ref,
                     int nthreads,
                     float* out,
                     uint64_t out_len) {
    return guarded([&] {
        auto fold = loki::algorithms::compute_brute_fold<float>(
            std::span<const float>(ts_e, nsamps),
            std::span<const float>(ts_v, nsamps),
            std::span<const double>(freqs, nfreqs), segment_len, nbins, tsamp,
            t_ref, nthreads);
        if (fold.size() != out_len) {
            throw std::runtime_error("lkref_brute_fold: output size mismatch");
        }
        std::memcpy(out, fold.data(), fold.size() * sizeof(float));
    });
}

int lkref_snr_boxcar_3d(const float* folds,
                        uint64_t nprofiles,
                        uint64_t nbins,
                        const uint64_t* widths,
                        uint64_t nwidths,
                        int nthreads,
                        float* scores) {
    return guarded([&] {
        std::vector<loki::SizeType> w(widths, widths + nwidths);
        loki::detection::snr_boxcar_3d(
            std::span<const float>(folds, nprofiles * 2 * nbins), w,
            std::span<float>(scores, nprofiles * nwidths), nprofiles, nbins,
            nthreads);
    });
}

int lkref_snr_boxcar_3d_max(const float* folds,
                            uint64_t nprofiles,
                            uint64_t nbins,
                            const uint64_t* widths,
                            uint64_t nwidths,
                            int nthreads,
                            float* scores) {
    return guarded([&] {
        std::vector<loki::SizeType> w(widths, widths + nwidths);
        loki::detection::snr_boxcar_3d_max(
            std::span<const float>(folds, nprofiles * 2 * nbins), w,
            std::span<float>(scores, nprofiles), nprofiles, nbins, nthreads);
    });
}

int lkref_box_widths(uint64_t nbins,
                     double ducy_max,
                     double wtsp,
                     uint64_t* out,
                     uint64_t max_out,
                     uint64_t* n_out) {
    return guarded([&] {
        auto w = loki::detection::generate_box_width_trials(nbins, ducy_max, wtsp);
        if (w.size() > max_out) {
            throw std::runtime_error("lkref_box_widths: output too small");
        }
        for (loki::SizeType i = 0; i < w.size(); ++i) {
            out[i] = w[i];
        }
        *n_out = w.size();
    });
}

float lkref_phase_idx(double proper_time, double freq, uint64_t nbins, double delay) {
    return loki::psr_utils::get_phase_idx(proper_time, freq, nbins, delay);
}

uint32_t lkref_phase_idx_uint(double proper_time,
                              double freq,
                              uint64_t nbins,
                              double delay) {
    return loki::psr_utils::get_phase_idx_uint(proper_time, freq, nbins, delay);
}

// detection::snr_boxcar_threshold_with_cache (lib/score.cpp:434-462) of n
// 2-D profiles, thresholds[i] for profile i: out[i] = 1 if some width's
// S/N / stdnoise > thresholds[i].
int lkref_snr_threshold(const float* profiles, uint64_t n, uint64_t nbins,
                        const uint64_t* widths, uint64_t nwidths, const float* thresholds,
                        float stdnoise, uint8_t* out) {
    return guarded([&] {
        std::vector<loki::SizeType> w(widths, widths + nwidths);
        loki::detection::BoxcarWidthsCache cache(w, nbins);
        for (uint64_t i = 0; i < n; ++i) {
            out[i] = loki::detection::snr_boxcar_threshold_with_cache(
                         std::span<const float>(profiles + i * nbins, nbins), nbins, cache,
                         thresholds[i], stdnoise)
                         ? 1
                         : 0;
        }
    });
}

// ---- pruning leaf step ------------------------------------------------------

// MiddleOutScheme of (nsegments, ref_idx, tsegment) at one level: out[0] =
// segment index, out[1..2] = get_coord, out[3..4] = get_current_coord,
// out[5..6] = get_segment_coord.
int lkref_middle_out(uint64_t nsegments, uint64_t ref_idx, double tsegment, uint64_t level,
                     double* out) {
    return guarded([&] {
        const loki::psr_utils::MiddleOutScheme sc(nsegments, ref_idx, tsegment);
        out[0]         = static_cast<double>(sc.get_segment_idx(level));
        const auto c   = sc.get_coord(level);
        const auto cur = sc.get_current_coord(level);
        const auto seg = sc.get_segment_coord(level);
        out[1] = c.first;
        out[2] = c.second;
        out[3] = cur.first;
        out[4] = cur.second;
        out[5] = seg.first;
        out[6] = seg.second;
    });
}

static loki::search::PulsarSearchConfig make_cfg_prune(const lkref_cfg* c, int conservative) {
    std::vector<loki::ParamLimit> lims(c->nparams);
    for (uint32_t i = 0; i < c->nparams; ++i) {
        lims[i] = {.min = c->limits[2 * i], .max = c->limits[(2 * i) + 1]};
    }
    std::optional<loki::SizeType> bb;
    std::optional<loki::SizeType> bf;
    if (c->bseg_brute != 0) {
        bb = c->bseg_brute;
    }
    if (c->bseg_ffa != 0) {
        bf = c->bseg_ffa;
    }
    return {c->nsamps, c->tsamp, c->nbins, c->eta, lims, c->ducy_max, c->wtsp,
            /*use_fourier=*/false, c->nthreads,
            /*max_process_memory_gb=*/8.0, /*octave_scale=*/2.0,
            /*nbins_max=*/1024, /*nbins_min_lossy_bf=*/64, bb, bf,
            /*snr_min=*/5.0, /*max_passing_candidates=*/1U << 22U,
            /*prune_poly_order=*/3, /*p_orb_min=*/1e-5, /*m_c_max=*/10.0,
            /*m_p_min=*/1.4, /*minimum_snap_cells=*/5.0, conservative != 0};
}

// Seed leaves of the final FFA level ([ncoords, nparams + 2, 2] doubles).
int lkref_taylor_seed(const lkref_cfg* c, double* leaves_out, uint64_t cap, uint64_t* n_out) {
    return guarded([&] {
        const auto cfg = make_cfg_prune(c, 0);
        const loki::plans::FFAPlan<float> plan(cfg);
        std::span<double> out(leaves_out, cap * (c->nparams + 2) * 2);
        *n_out = loki::core::poly_taylor_seed(plan.get_param_counts().back(),
                                              plan.get_dparams_actual().back(),
                                              cfg.get_param_limits(), out, {0.0, 0.0},
                                              c->nparams);
    });
}

// Branch n parent leaves. leaves_out must hold n * branch_max leaves.
int lkref_taylor_branch(const double* leaves_in, uint64_t n, uint32_t nparams, double t_cur,
                        double scale_cur, uint64_t nbins, double eta, uint64_t branch_max,
                        double* leaves_out, uint64_t* origins_out, uint64_t* n_out) {
    return guarded([&] {
        const uint64_t stride = (nparams + 2) * 2;
        loki::memory::BranchingWorkspace ws(n, branch_max, nparams);
        std::span<const double> in(leaves_in, n * stride);
        std::span<double> out(leaves_out, n * branch_max * stride);
        std::span<loki::SizeType> org(reinterpret_cast<loki::SizeType*>(origins_out),
                                      n * branch_max);
        *n_out = loki::core::poly_taylor_branch_batch(in, out, org, {t_cur, scale_cur}, nbins,
                                                      eta, branch_max, n, nparams, ws);
    });
}

// Resolve n leaves against the final FFA level of the configuration.
// coords = {t_add, s_add, t_cur, s_cur, t_init, s_init}.
int lkref_taylor_resolve(const lkref_cfg* c, const double* leaves, uint64_t n,
                         const double* coords, uint64_t* param_idx, float* phase_shift) {
    return guarded([&] {
        const auto cfg = make_cfg_prune(c, 0);
        const loki::plans::FFAPlan<float> plan(cfg);
        const auto& counts = plan.get_param_counts().back();
        const uint64_t stride = (c->nparams + 2) * 2;
        loki::core::poly_taylor_resolve_batch(
            std::span<const double>(leaves, n * stride),
            std::span<loki::SizeType>(reinterpret_cast<loki::SizeType*>(param_idx), n),
            std::span<float>(phase_shift, n), cfg.get_param_limits(), {coords[0], coords[1]},
            {coords[2], coords[3]}, {coords[4], coords[5]}, counts[c->nparams - 2],
            counts[c->nparams - 1], c->nbins, n, c->nparams);
    });
}

// In-place transform of the leaves named by indices[0..n).
int lkref_taylor_transform(double* leaves, uint64_t n_leaves_total, const uint64_t* indices,
                           uint64_t n, uint32_t nparams, double t_next, double s_next,
                           double t_cur, double s_cur, int conservative) {
    return guarded([&] {
        const uint64_t stride = (nparams + 2) * 2;
        std::vector<loki::SizeType> idx(indices, indices + n);
        loki::core::poly_taylor_transform_batch(std::span<double>(leaves, n_leaves_total * stride),
                                                idx, {t_next, s_next}, {t_cur, s_cur}, n,
                                                nparams, conservative != 0);
    });
}

int lkref_shift_add_batch(const float* folds_tree, const uint64_t* indices_tree,
                          const float* folds_ffa, const uint64_t* indices_ffa,
                          const float* phase_shift, float* folds_out, uint64_t nbins,
                          uint64_t n_leaves, uint64_t physical_start_idx, uint64_t capacity) {
    return guarded([&] {
        std::vector<float> tmp(2 * nbins);
        loki::kernels::shift_add_linear_batch(
            folds_tree, reinterpret_cast<const loki::SizeType*>(indices_tree), folds_ffa,
            reinterpret_cast<const loki::SizeType*>(indices_ffa), phase_shift, folds_out,
            tmp.data(), nbins, n_leaves, physical_start_idx, capacity);
    });
}

int lkref_score_filter(const float* folds, uint64_t n, uint64_t nbins, const uint64_t* widths,
                       uint64_t nwidths, float threshold, float* scores, uint64_t* indices,
                       uint64_t* n_pass) {
    return guarded([&] {
        std::vector<loki::SizeType> w(widths, widths + nwidths);
        loki::detection::BoxcarWidthsCache cache(w, nbins);
        *n_pass = loki::detection::score_and_filter_max_with_cache(
            std::span<const float>(folds, n * 2 * nbins), std::span<float>(scores, n),
            std::span<loki::SizeType>(reinterpret_cast<loki::SizeType*>(indices), n),
            threshold, n, nbins, cache);
    });
}

// EPMultiPass's branch_max: max(ceil(2 * max branching pattern), 32).
int lkref_branch_max(const lkref_cfg* c, int conservative, uint64_t* out) {
    return guarded([&] {
        const auto cfg = make_cfg_prune(c, conservative);
        const loki::plans::FFAPlan<float> plan(cfg);
        const auto bp = plan.get_branching_pattern("taylor");
        const auto mx = *std::ranges::max_element(bp);
        *out = std::max(static_cast<loki::SizeType>(std::ceil(mx * 2)), loki::SizeType{32});
    });
}

// FFAPlan::get_branching_pattern("taylor", ref_seg) (lib/plans.cpp:219-259).
int lkref_branching_pattern(const lkref_cfg* c, int conservative, uint64_t ref_seg,
                            double* out, uint64_t max_out, uint64_t* n_out) {
    return guarded([&] {
        const auto cfg = make_cfg_prune(c, conservative);
        const loki::plans::FFAPlan<float> plan(cfg);
        const auto bp = plan.get_branching_pattern("taylor", ref_seg);
        *n_out = bp.size();
        std::copy_n(bp.begin(), std::min<uint64_t>(bp.size(), max_out), out);
    });
}

// ---- Chebyshev basis (lib/chebyshev.cpp) -----------------------------------

int lkref_taylor_to_cheby(double* leaves, uint64_t n, uint32_t nparams, double t_init,
                          double s_init) {
    return guarded([&] {
        loki::core::poly_taylor_to_cheby_batch(
            std::span<double>(leaves, n * (nparams + 2) * 2), {t_init, s_init}, n, nparams);
    });
}

int lkref_cheby_to_taylor(double* leaves, uint64_t n, uint32_t nparams, double t_report,
                          double s_report) {
    return guarded([&] {
        loki::core::poly_cheby_to_taylor_batch(
            std::span<double>(leaves, n * (nparams + 2) * 2), {t_report, s_report}, n, nparams);
    });
}

// Branch n parents; leaves_in is transformed in place (coord_prev ->
// coord_cur) as the reference does. leaves_out must hold n * branch_max.
int lkref_cheby_branch(double* leaves_in, uint64_t n, uint32_t nparams, double t_cur,
                       double s_cur, double t_prev, double s_prev, uint64_t nbins, double eta,
                       uint64_t branch_max, double* leaves_out, uint64_t* origins_out,
                       uint64_t* n_out) {
    return guarded([&] {
        const uint64_t stride = (nparams + 2) * 2;
        loki::memory::BranchingWorkspace ws(n, branch_max, nparams);
        std::span<double> in(leaves_in, n * stride);
        std::span<double> out(leaves_out, n * branch_max * stride);
        std::span<loki::SizeType> org(reinterpret_cast<loki::SizeType*>(origins_out),
                                      n * branch_max);
        *n_out = loki::core::poly_chebyshev_branch_batch(in, out, org, {t_cur, s_cur},
                                                         {t_prev, s_prev}, nbins, eta,
                                                         branch_max, n, nparams, ws);
    });
}

// coords = {t_add, s_add, t_cur, s_cur, t_init, s_init}.
int lkref_cheby_resolve(const lkref_cfg* c, const double* leaves, uint64_t n,
                        const double* coords, uint64_t* param_idx, float* phase_shift) {
    return guarded([&] {
        const auto cfg = make_cfg_prune(c, 0);
        const loki::plans::FFAPlan<float> plan(cfg);
        const auto& counts = plan.get_param_counts().back();
        const uint64_t stride = (c->nparams + 2) * 2;
        loki::core::poly_chebyshev_resolve_batch(
            std::span<const double>(leaves, n * stride),
            std::span<loki::SizeType>(reinterpret_cast<loki::SizeType*>(param_idx), n),
            std::span<float>(phase_shift, n), cfg.get_param_limits(), {coords[0], coords[1]},
            {coords[2], coords[3]}, {coords[4], coords[5]}, counts[c->nparams - 2],
            counts[c->nparams - 1], c->nbins, n, c->nparams);
    });
}

int lkref_cheby_transform(double* leaves, uint64_t n_leaves_total, const uint64_t* indices,
                          uint64_t n, uint32_t nparams, double t_next, double s_next,
                          double t_cur, double s_cur) {
    return guarded([&] {
        const uint64_t stride = (nparams + 2) * 2;
        std::vector<loki::SizeType> idx(indices, indices + n);
        loki::core::poly_chebyshev_transform_batch(
            std::span<double>(leaves, n_leaves_total * stride), idx, {t_next, s_next},
            {t_cur, s_cur}, n, nparams);
    });
}

// FFAPlan::get_branching_pattern(basis, ref_seg), basis 0 taylor / 1 chebyshev.
int lkref_branching_pattern_basis(const lkref_cfg* c, int basis, int conservative,
                                  uint64_t ref_seg, double* out, uint64_t max_out,
                                  uint64_t* n_out) {
    return guarded([&] {
        const auto cfg = make_cfg_prune(c, conservative);
        const loki::plans::FFAPlan<float> plan(cfg);
        const auto bp = plan.get_branching_pattern(basis == 1 ? "chebyshev" : "taylor", ref_seg);
        *n_out = bp.size();
        std::copy_n(bp.begin(), std::min<uint64_t>(bp.size(), max_out), out);
    });
}

// Per-level statistics (cands::PruneStats fields).
struct lkref_prune_stats {
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
};

// One pruning run for ref_seg over the FFA fold of the final level
// ([nsegments, ncoords, 2, nbins]): seed, then up to n_iters levels (each
// uses thresholds[level - 1]). stats receives one row for the seed and one
// per level run; the final tree is copied out in logical order.
static int prune_run_basis(const char* basis, const lkref_cfg* c, int conservative,
                           const float* ffa_fold, uint64_t ffa_fold_len, const float* thresholds,
                           uint64_t n_thresholds, uint64_t ref_seg, uint64_t max_sugg,
                           uint64_t batch_size, uint64_t branch_max, uint64_t n_iters,
                           lkref_prune_stats* stats, uint64_t* n_stats, double* leaves_out,
                           float* folds_out, float* scores_out, uint64_t cap_out,
                           uint64_t* n_out, int finalize = 0, float* scores_ep_out = nullptr);

int lkref_prune_run(const lkref_cfg* c, int conservative, const float* ffa_fold,
                    uint64_t ffa_fold_len, const float* thresholds, uint64_t n_thresholds,
                    uint64_t ref_seg, uint64_t max_sugg, uint64_t batch_size,
                    uint64_t branch_max, uint64_t n_iters, lkref_prune_stats* stats,
                    uint64_t* n_stats, double* leaves_out, float* folds_out, float* scores_out,
                    uint64_t cap_out, uint64_t* n_out) {
    return prune_run_basis("taylor", c, conservative, ffa_fold, ffa_fold_len, thresholds,
                           n_thresholds, ref_seg, max_sugg, batch_size, branch_max, n_iters,
                           stats, n_stats, leaves_out, folds_out, scores_out, cap_out, n_out);
}

// FFARegionPlanner<float> (lib/regions.cpp:157-514) on a base configuration
// with the given planner knobs. Per chunk, 6 doubles: f_min, f_max (the
// drift-widened frequency limits), nbins, eta, bseg_brute, bseg_ffa. stats_out
// (5 doubles): max buffer size, max coord size, max ncoords, max FFA levels,
// get_freq_sweep_memory_usage() in GB (the device model when use_gpu).
}  // extern "C"

template <class FoldType>
static int region_plan(const lkref_cfg* c, double max_memory_gb, double octave_scale,
                       uint64_t nbins_max, uint64_t max_passing, int use_gpu, bool use_fourier,
                       double* chunks_out, uint64_t cap, uint64_t* n_out, double* stats_out) {
    return guarded([&] {
        std::vector<loki::ParamLimit> lims(c->nparams);
        for (uint32_t i = 0; i < c->nparams; ++i) {
            lims[i] = {.min = c->limits[2 * i], .max = c->limits[(2 * i) + 1]};
        }
        std::optional<loki::SizeType> bb;
        std::optional<loki::SizeType> bf;
        if (c->bseg_brute != 0) {
            bb = c->bseg_brute;
        }
        if (c->bseg_ffa != 0) {
            bf = c->bseg_ffa;
        }
        const loki::search::PulsarSearchConfig cfg(
            c->nsamps, c->tsamp, c->nbins, c->eta, lims, c->ducy_max, c->wtsp,
            use_fourier, c->nthreads, max_memory_gb, octave_scale, nbins_max,
            /*nbins_min_lossy_bf=*/64, bb, bf, /*snr_min=*/5.0, max_passing);
        const loki::regions::FFARegionPlanner<FoldType> planner(cfg, use_gpu != 0);
        const auto& cfgs = planner.get_cfgs();
        *n_out = cfgs.size();
        for (std::size_t i = 0; i < cfgs.size() && i < cap; ++i) {
            const auto pl = cfgs[i].get_param_limits();
            double* row = chunks_out + (6 * i);
            row[0] = pl.back().min;
            row[1] = pl.back().max;
            row[2] = static_cast<double>(cfgs[i].get_nbins());
            row[3] = cfgs[i].get_eta();
            row[4] = static_cast<double>(cfgs[i].get_bseg_brute());
            row[5] = static_cast<double>(cfgs[i].get_bseg_ffa());
        }
        const auto& st = planner.get_stats();
        stats_out[0] = static_cast<double>(st.get_max_buffer_size());
        stats_out[1] = static_cast<double>(st.get_max_coord_size());
        stats_out[2] = static_cast<double>(st.get_max_ncoords());
        stats_out[3] = static_cast<double>(st.get_max_ffa_levels());
        stats_out[4] = static_cast<double>(st.get_freq_sweep_memory_usage());
    });
}

extern "C" {

int lkref_region_plan(const lkref_cfg* c, double max_memory_gb, double octave_scale,
                      uint64_t nbins_max, uint64_t max_passing, int use_gpu, double* chunks_out,
                      uint64_t cap, uint64_t* n_out, double* stats_out) {
    return region_plan<float>(c, max_memory_gb, octave_scale, nbins_max, max_passing, use_gpu, false,
                              chunks_out, cap, n_out, stats_out);
}

// The planner of a given fold type (0 float, 1 ComplexType) on a configuration
// with the given use_fourier.
int lkref_region_plan_typed(const lkref_cfg* c, double max_memory_gb, double octave_scale,
                            uint64_t nbins_max, uint64_t max_passing, int use_gpu, int complex_fold,
                            int use_fourier, double* chunks_out, uint64_t cap, uint64_t* n_out,
                            double* stats_out) {
    return complex_fold != 0
               ? region_plan<loki::ComplexType>(c, max_memory_gb, octave_scale, nbins_max, max_passing,
                                                use_gpu, use_fourier != 0, chunks_out, cap, n_out,
                                                stats_out)
               : region_plan<float>(c, max_memory_gb, octave_scale, nbins_max, max_passing, use_gpu,
                                    use_fourier != 0, chunks_out, cap, n_out, stats_out);
}

// The same run with poly_basis "taylor" (basis 0) or "chebyshev" (basis 1).
int lkref_prune_run_basis(int basis, const lkref_cfg* c, int conservative,
                          const float* ffa_fold, uint64_t ffa_fold_len, const float* thresholds,
                          uint64_t n_thresholds, uint64_t ref_seg, uint64_t max_sugg,
                          uint64_t batch_size, uint64_t branch_max, uint64_t n_iters,
                          lkref_prune_stats* stats, uint64_t* n_stats, double* leaves_out,
                          float* folds_out, float* scores_out, uint64_t cap_out,
                          uint64_t* n_out) {
    return prune_run_basis(basis == 1 ? "chebyshev" : "taylor", c, conservative, ffa_fold,
                           ffa_fold_len, thresholds, n_thresholds, ref_seg, max_sugg, batch_size,
                           branch_max, n_iters, stats, n_stats, leaves_out, folds_out,
                           scores_out, cap_out, n_out);
}

// A whole EPMultiPass run for one ref_seg as PruneImpl::run does it: the
// levels, then the survivors ascended to the middle of the data (folds and
// scores over every segment so far; scores_ep = the scores before) and
// reported there (prune.cpp:136-139,228-334).
int lkref_prune_run_full(int basis, const lkref_cfg* c, int conservative, const float* ffa_fold,
                         uint64_t ffa_fold_len, const float* thresholds, uint64_t n_thresholds,
                         uint64_t ref_seg, uint64_t max_sugg, uint64_t batch_size,
                         uint64_t branch_max, uint64_t n_iters, lkref_prune_stats* stats,
                         uint64_t* n_stats, double* leaves_out, float* folds_out,
                         float* scores_out, float* scores_ep_out, uint64_t cap_out,
                         uint64_t* n_out) {
    return prune_run_basis(basis == 1 ? "chebyshev" : "taylor", c, conservative, ffa_fold,
                           ffa_fold_len, thresholds, n_thresholds, ref_seg, max_sugg, batch_size,
                           branch_max, n_iters, stats, n_stats, leaves_out, folds_out,
                           scores_out, cap_out, n_out, 1, scores_ep_out);
}

static int prune_run_basis(const char* basis, const lkref_cfg* c, int conservative,
                           const float* ffa_fold, uint64_t ffa_fold_len, const float* thresholds,
                           uint64_t n_thresholds, uint64_t ref_seg, uint64_t max_sugg,
                           uint64_t batch_size, uint64_t branch_max, uint64_t n_iters,
                           lkref_prune_stats* stats, uint64_t* n_stats, double* leaves_out,
                           float* folds_out, float* scores_out, uint64_t cap_out,
                           uint64_t* n_out, int finalize, float* scores_ep_out) {
    return guarded([&] {
        using loki::SizeType;
        const auto cfg = make_cfg_prune(c, conservative);
        const loki::plans::FFAPlan<float> plan(cfg);
        const SizeType nsegments = plan.get_nsegments().back();
        const double tseg        = plan.get_tsegments().back();
        const SizeType nparams   = cfg.get_nparams();
        const SizeType nbins     = cfg.get_nbins();
        auto funcs = loki::core::create_prune_dp_functs<float>(
            basis, plan.get_param_counts().back(), plan.get_dparams_actual().back(),
            nsegments, tseg, cfg, batch_size, branch_max);
        loki::memory::EPWorkspace<float> ws(batch_size, branch_max, max_sugg,
                                            plan.get_ncoords().back(), nparams, nbins,
                                            nsegments);
        auto& world_tree = ws.world_tree;
        auto& prune_ws   = ws.prune;
        auto& branch_ws  = ws.branch;
        const std::span<const float> ffa(ffa_fold, ffa_fold_len);

        // initialize (prune.cpp:181-226)
        world_tree.reset();
        const loki::psr_utils::MiddleOutScheme snail(nsegments, ref_seg, tseg);
        const auto fold_segment = funcs->load_segment(ffa, snail.get_ref_idx());
        const auto coord_init0  = snail.get_coord(0);
        const SizeType n_seed   = plan.get_ncoords().back();
        funcs->seed(fold_segment, ws.seed_leaves, ws.seed_scores, coord_init0);
        world_tree.add_initial(ws.seed_leaves, fold_segment, ws.seed_scores, n_seed);
        SizeType ns = 0;
        stats[ns++] = {0, snail.get_segment_idx(0), world_tree.get_size(),
                       world_tree.get_size(), world_tree.get_size(), world_tree.get_size(),
                       0.0F, world_tree.get_score_min(), world_tree.get_score_max(), 0.0F};

        // levels (prune.cpp:429-620)
        const SizeType levels = std::min<SizeType>(nsegments - 1, n_iters);
        for (SizeType prune_level = 1; prune_level <= levels; ++prune_level) {
            if (prune_level > n_thresholds) {
                throw std::runtime_error("Pruning complete - exceeded threshold scheme length");
            }
            world_tree.prepare_in_place_update();
            const SizeType seg_idx_cur = snail.get_segment_idx(prune_level);
            const float threshold      = thresholds[prune_level - 1];
            const SizeType n_branches  = world_tree.get_size_old();
            SizeType n_leaves = 0, n_leaves_phy = 0;
            float score_min = std::numeric_limits<float>::max();
            float score_max = std::numeric_limits<float>::lowest();

            const auto coord_init = snail.get_coord(0);
            const auto coord_prev = snail.get_coord(prune_level - 1);
            const auto coord_next = snail.get_coord(prune_level);
            const auto coord_cur  = snail.get_current_coord(prune_level);
            const auto coord_add  = snail.get_segment_coord(prune_level);
            const auto ffa_fold_segment = funcs->load_segment(ffa, seg_idx_cur);
            auto current_threshold = threshold;
            const SizeType bsize = std::max<SizeType>(1, std::min(batch_size, n_branches));
            SizeType total_processed = 0;
            while (total_processed < n_branches) {
                const SizeType remaining       = n_branches - total_processed;
                const SizeType this_batch_size = std::min(bsize, remaining);
                auto [leaves_tree_span, current_batch_size] =
                    world_tree.get_leaves_span(this_batch_size);
                if (current_batch_size == 0) {
                    throw std::runtime_error("Loaded batch size is 0");
                }
                total_processed += current_batch_size;
                const auto n_leaves_batch = funcs->branch(
                    leaves_tree_span, prune_ws.branched_leaves, prune_ws.branched_indices,
                    coord_cur, coord_prev, current_batch_size, branch_ws);
                n_leaves += n_leaves_batch;
                if (n_leaves_batch == 0) {
                    world_tree.consume_read(current_batch_size);
                    continue;
                }
                if (n_leaves_batch > prune_ws.max_branched_leaves) {
                    throw std::runtime_error("Branch factor exceeded workspace size");
                }
                const auto n_valid = funcs->validate(prune_ws.branched_leaves,
                                                     prune_ws.branched_indices, coord_cur,
                                                     n_leaves_batch);
                n_leaves_phy += n_valid;
                if (n_valid == 0) {
                    world_tree.consume_read(current_batch_size);
                    continue;
                }
                funcs->resolve(prune_ws.branched_leaves, prune_ws.branched_param_idx,
                               prune_ws.branched_phase_shift, coord_add, coord_cur,
                               coord_init, n_valid);
                funcs->shift_add(world_tree.get_folds(), prune_ws.branched_indices,
                                 ffa_fold_segment, prune_ws.branched_param_idx,
                                 prune_ws.branched_phase_shift, prune_ws.branched_folds,
                                 n_valid, world_tree.get_physical_start_idx(),
                                 world_tree.get_capacity());
                const SizeType n_pass = funcs->score_and_filter(
                    prune_ws.branched_folds, prune_ws.branched_scores,
                    prune_ws.branched_indices, current_threshold, n_valid);
                const auto sc = std::span<const float>(prune_ws.branched_scores).first(n_valid);
                const auto [mn, mx] = std::ranges::minmax_element(sc);
                score_min = std::min(score_min, *mn);
                score_max = std::max(score_max, *mx);
                if (n_pass == 0) {
                    world_tree.consume_read(current_batch_size);
                    continue;
                }
                funcs->transform(prune_ws.branched_leaves, prune_ws.branched_indices,
                                 coord_next, coord_cur, n_pass);
                current_threshold = world_tree.add_batch_scattered(
                    prune_ws.branched_leaves, prune_ws.branched_folds,
                    prune_ws.branched_scores, prune_ws.branched_indices, current_threshold,
                    n_pass);
                world_tree.consume_read(current_batch_size);
            }
            world_tree.finalize_in_place_update();
            stats[ns++] = {prune_level, seg_idx_cur, n_branches, n_leaves, n_leaves_phy,
                           world_tree.get_size(), threshold, score_min, score_max, 0.0F};
            if (world_tree.get_size() == 0) {
                break;
            }
        }
        *n_stats = ns;

        // ascend_survivors_batched + report_survivors (prune.cpp:136-139,
        // 228-334): survivors of a run that kept any are ascended to the
        // middle of the data and reported there.
        if (finalize != 0 && world_tree.get_size() > 0) {
            const SizeType prune_level = ns - 1;
            const auto coord_mid = snail.get_coord(prune_level);
            const auto [idx_segments, coord_segments] =
                snail.get_segment_coords_so_far(prune_level);
            const SizeType n_surv  = world_tree.get_size();
            const SizeType cap_b   = std::max(SizeType{1}, std::min(batch_size, n_surv));
            const SizeType lstride = world_tree.get_leaves_stride();
            const SizeType fstride = world_tree.get_folds_stride();
            auto lv = world_tree.get_leaves_circular_view();
            auto fv = world_tree.get_folds_circular_view();
            auto sv = world_tree.get_scores_circular_view();
            auto ev = world_tree.get_scores_ep_circular_view();
            auto region = [&](std::span<double> l, std::span<float> f, std::span<float> sc,
                              std::span<float> ep) {
                const SizeType nreg = l.size() / lstride;
                for (SizeType off = 0; off < nreg; off += cap_b) {
                    const SizeType chunk = std::min(cap_b, nreg - off);
                    funcs->ascend(ffa, l.subspan(off * lstride, chunk * lstride),
                                  f.subspan(off * fstride, chunk * fstride),
                                  sc.subspan(off, chunk), ep.subspan(off, chunk), idx_segments,
                                  coord_segments, coord_mid, prune_ws.branched_param_idx,
                                  prune_ws.branched_phase_shift, chunk);
                }
            };
            region(lv.first, fv.first, sv.first, ev.first);
            region(lv.second, fv.second, sv.second, ev.second);
            const SizeType n1 = lv.first.size() / lstride;
            const SizeType n2 = lv.second.size() / lstride;
            funcs->report(lv.first, coord_mid, n1);
            if (n2 > 0) {
                funcs->report(lv.second, coord_mid, n2);
            }
        }

        // final tree in logical order
        const SizeType n = world_tree.get_size();
        *n_out = n;
        if (n > cap_out) {
            return;
        }
        const SizeType ls = world_tree.get_leaves_stride();
        const SizeType fs = world_tree.get_folds_stride();
        const auto lv = world_tree.get_leaves_circular_view();
        const auto fv = world_tree.get_folds_circular_view();
        const auto sv = world_tree.get_scores_circular_view();
        std::copy(lv.first.begin(), lv.first.end(), leaves_out);
        std::copy(lv.second.begin(), lv.second.end(), leaves_out + lv.first.size());
        std::copy(fv.first.begin(), fv.first.end(), folds_out);
        std::copy(fv.second.begin(), fv.second.end(), folds_out + fv.first.size());
        std::copy(sv.first.begin(), sv.first.end(), scores_out);
        std::copy(sv.second.begin(), sv.second.end(), scores_out + sv.first.size());
        if (scores_ep_out != nullptr) {
            const auto ev = world_tree.get_scores_ep_circular_view();
            std::copy(ev.first.begin(), ev.first.end(), scores_ep_out);
            std::copy(ev.second.begin(), ev.second.end(), scores_ep_out + ev.first.size());
        }
        (void)ls;
        (void)fs;
    });
}

// ---- DynamicThresholdScheme ---------------------------------------------------

int lkref_dts_thresholds(float snr_start, float snr_final, uint64_t n, float* out) {
    return guarded([&] {
        const auto t = loki::detection::detail::compute_thresholds(snr_start, snr_final, n);
        std::copy(t.begin(), t.end(), out);
    });
}

int lkref_dts_probs(uint64_t n, float prob_min, float* out) {
    return guarded([&] {
        const auto p = loki::detection::detail::compute_probs(n, prob_min);
        std::copy(p.begin(), p.end(), out);
    });
}

int lkref_dts_profile(uint64_t nbins, float ducy, float center, float* out) {
    return guarded([&] {
        const auto p = loki::simulation::generate_folded_profile(nbins, ducy, center);
        std::copy(p.begin(), p.end(), out);
    });
}

int lkref_dts_bound(uint64_t nstages, float snr_bound, float* out) {
    return guarded([&] {
        const auto b = loki::detection::detail::bound_scheme(nstages, snr_bound);
        std::copy(b.begin(), b.end(), out);
    });
}

int lkref_dts_neighbours(const uint64_t* idx, uint64_t n, uint64_t target, uint64_t num, uint64_t* out,
                         uint64_t* n_out) {
    return guarded([&] {
        const auto r = loki::utils::find_neighbouring_indices(std::span<const loki::SizeType>(idx, n), target, num);
        std::copy(r.begin(), r.end(), out);
        *n_out = r.size();
    });
}

int64_t lkref_dts_lower_bin(const float* range, uint64_t n, float v) {
    return loki::utils::find_lower_bin_index(std::span<const float>(range, n), v);
}

using loki::detection::State;
static_assert(sizeof(State) == 44, "State layout");

int lkref_dts_gen_next(const void* state, float threshold, float s0, float s1, float nbranches, void* out) {
    return guarded([&] {
        State st;
        std::memcpy(&st, state, sizeof(State));
        const State n = st.gen_next(threshold, s0, s1, nbranches);
        std::memcpy(out, &n, sizeof(State));
    });
}

int lkref_dts_best_path(const void* states, uint64_t nstages, const float* thresholds, uint64_t nthresholds,
                        const float* probs, uint64_t nprobs, float min_pd, float* out, uint64_t* n_out) {
    return guarded([&] {
        std::vector<State> st(nstages * nthresholds * nprobs);
        std::memcpy(st.data(), states, st.size() * sizeof(State));
        const auto r = loki::detection::detail::get_best_path_thresholds(
            st, std::span<const float>(thresholds, nthresholds), std::span<const float>(probs, nprobs), nstages,
            nthresholds, nprobs, min_pd);
        std::copy(r.begin(), r.end(), out);
        *n_out = r.size();
    });
}

namespace {

uint32_t dts_philox_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, int q) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    const uint32_t w[4] = {c0, c1, c2, c3};
    return w[q];
}

// The stream of one (transition, hypothesis): generate_impl / uniform_index
// of ThreadLocalNormalRNG (lib/loki/math.hpp:267-285,363-390) on counter
// words instead of a thread-local PCG32.
struct CounterNormal {
    const std::vector<float>* lut;
    uint32_t k0, k1, tid2, stage;
    float normal(uint32_t i, uint32_t j) const {
        const uint32_t r = dts_philox_word(i, j / 4, tid2, stage, k0, k1, static_cast<int>(j % 4));
        constexpr float kInvU32 = 1.0F / static_cast<float>(std::numeric_limits<uint32_t>::max());
        const auto max_idx = static_cast<float>(lut->size() - 2);
        const float u_scaled = static_cast<float>(r) * kInvU32 * max_idx;
        const auto idx = static_cast<loki::SizeType>(u_scaled);
        const float frac = u_scaled - static_cast<float>(idx);
        const float z = std::fma(frac, (*lut)[idx + 1] - (*lut)[idx], (*lut)[idx]);
        return std::fma(z, 1.0F, 0.0F);
    }
    uint32_t uniform_index(uint32_t i, uint32_t max_value) const {
        const uint64_t range = static_cast<uint64_t>(max_value) + 1ULL;
        const uint64_t t = (1ULL << 32U) % range;
        uint64_t m = 0;
        for (uint32_t call = 0; call < 2; ++call) {
            for (int q = 0; q < 4; ++q) {
                m = static_cast<uint64_t>(dts_philox_word(i, 0xFFFFFFFFu - call, tid2, stage, k0, k1, q)) * range;
                const auto l = static_cast<uint32_t>(m);
                if (l >= range || l >= t) {
                    return static_cast<uint32_t>(m >> 32U);
                }
            }
        }
        return static_cast<uint32_t>(m >> 32U);
    }
};

// simulate_score_prune_fused (lib/thresholds.cpp:358-431) with the stream above.
uint32_t dts_sim(const std::vector<float>& in, uint32_t n_in, std::span<const float> profile, float bias,
                 const CounterNormal& rng, uint32_t ntrials, uint32_t nbins,
                 loki::detection::BoxcarWidthsCache& cache, float threshold, float var_in,
                 std::vector<float>& out) {
    std::vector<float> prof(nbins);
    for (uint32_t j = 0; j < nbins; ++j) {
        prof[j] = profile[j] * bias;
    }
    const float stdnoise = std::sqrt(var_in + 1.0F);
    uint32_t n = 0;
    for (uint32_t i = 0; i < ntrials; ++i) {
        const uint32_t src = (i < n_in) ? i : rng.uniform_index(i, n_in - 1);
        float* o = out.data() + static_cast<uint64_t>(n) * nbins;
        for (uint32_t j = 0; j < nbins; ++j) {
            o[j] = in[static_cast<uint64_t>(src) * nbins + j] + rng.normal(i, j) + prof[j];
        }
        if (loki::detection::snr_boxcar_threshold_with_cache(std::span<const float>(o, nbins), nbins, cache,
                                                             threshold, stdnoise)) {
            ++n;
        }
    }
    return n;
}

} // namespace

// init_states + run / run_segment (lib/thresholds.cpp:748-907), sequential,
// over the reference's own pieces; guess: the guess path (norm_isf needs
// Boost.Math, absent here), lut: the normal quantile table; the first
// stages_run stages (0: all).
int lkref_dts_run(const float* branching, uint64_t nstages, float ref_ducy, uint64_t nbins, uint64_t ntrials,
                  uint64_t nprobs, float prob_min, float snr_final, uint64_t nthresholds, float ducy_max, float wtsp,
                  float beam_width, uint64_t seed, uint64_t thres_neigh, const float* guess, const float* lut_in,
                  uint64_t stages_run, void* states_out) {
    return guarded([&] {
        const std::vector<float> bp(branching, branching + nstages);
        const auto profile = loki::simulation::generate_folded_profile(nbins, ref_ducy);
        const auto thresholds = loki::detection::detail::compute_thresholds(0.1F, snr_final, nthresholds);
        const auto probs = loki::detection::detail::compute_probs(nprobs, prob_min);
        const auto widths = loki::detection::generate_box_width_trials(nbins, ducy_max, wtsp);
        loki::detection::BoxcarWidthsCache cache(widths, nbins);
        const float bias_snr = snr_final / static_cast<float>(std::sqrt(nstages + 1));
        const std::vector<float> lut(lut_in, lut_in + (1U << 17U) + 1U);
        const auto k0 = static_cast<uint32_t>(seed), k1 = static_cast<uint32_t>(seed >> 32U);
        auto beam = [&](uint64_t istage) {
            const float lower = std::max(0.0F, guess[istage] - beam_width);
            const float upper = std::min(thresholds.back(), guess[istage] + beam_width);
            std::vector<loki::SizeType> r;
            for (loki::SizeType i = 0; i < thresholds.size(); ++i) {
                if (thresholds[i] >= lower && thresholds[i] <= upper) {
                    r.push_back(i);
                }
            }
            return r;
        };
        const uint64_t ncell = nthresholds * nprobs;
        std::vector<State> states(nstages * ncell, State{});
        struct Folds {
            std::vector<float> f[2];
            uint32_t n[2] = {0, 0};
        };
        std::vector<Folds> cur(ncell), next(ncell);
        // initial folds: simulate_folds from zero folds, variance 0 + 1
        Folds init;
        for (int h = 0; h < 2; ++h) {
            init.f[h].resize(ntrials * nbins);
            init.n[h] = static_cast<uint32_t>(ntrials);
            const CounterNormal rng{&lut, k0, k1, static_cast<uint32_t>(h), 0U};
            const float bias = h == 0 ? 0.0F : bias_snr;
            for (uint32_t i = 0; i < ntrials; ++i) {
                for (uint32_t j = 0; j < nbins; ++j) {
                    init.f[h][i * nbins + j] = 0.0F + rng.normal(i, j) + profile[j] * bias;
                }
            }
        }
        const State initial = State::initial();
        float var_in = 1.0F;
        std::vector<loki::SizeType> beam_prev;
        std::vector<float> tmp[2] = {std::vector<float>(ntrials * nbins), std::vector<float>(ntrials * nbins)};
        const uint64_t s_run = (stages_run == 0 || stages_run > nstages) ? nstages : stages_run;
        for (uint64_t st = 0; st < s_run; ++st) {
            const auto beam_cur = beam(st);
            for (auto& f : next) {
                f.n[0] = f.n[1] = 0;
            }
            for (loki::SizeType ithres : beam_cur) {
                std::vector<loki::SizeType> neigh{0};
                if (st > 0) {
                    neigh = loki::utils::find_neighbouring_indices(beam_prev, ithres, thres_neigh);
                }
                for (loki::SizeType jthresh : neigh) {
                    for (uint64_t k = 0; k < (st == 0 ? 1 : nprobs); ++k) {
                        const uint64_t pc = jthresh * nprobs + k;
                        const State& ps = st == 0 ? initial : states[(st - 1) * ncell + pc];
                        const Folds& pf = st == 0 ? init : cur[pc];
                        if (ps.is_empty || pf.n[0] == 0 || pf.n[1] == 0) {
                            continue;
                        }
                        const auto tid = static_cast<uint32_t>(st == 0 ? ithres : (ithres * nthresholds + jthresh) * nprobs + k);
                        uint32_t m[2];
                        for (int h = 0; h < 2; ++h) {
                            const CounterNormal rng{&lut, k0, k1, 2 * tid + static_cast<uint32_t>(h),
                                                    static_cast<uint32_t>(st + 1)};
                            m[h] = dts_sim(pf.f[h], pf.n[h], profile, h == 0 ? 0.0F : bias_snr, rng,
                                           static_cast<uint32_t>(ntrials), static_cast<uint32_t>(nbins), cache,
                                           thresholds[ithres], var_in, tmp[h]);
                        }
                        const State ns = ps.gen_next(thresholds[ithres],
                                                     static_cast<float>(m[0]) / static_cast<float>(ntrials),
                                                     static_cast<float>(m[1]) / static_cast<float>(ntrials), bp[st]);
                        const auto ip = loki::utils::find_lower_bin_index(probs, ns.success_h1_cumul);
                        if (ip < 0 || ip >= static_cast<loki::IndexType>(nprobs)) {
                            continue;
                        }
                        const uint64_t cell = ithres * nprobs + static_cast<uint64_t>(ip);
                        State& ex = states[st * ncell + cell];
                        if (ex.is_empty || ns.complexity_cumul < ex.complexity_cumul) {
                            ex = ns;
                            for (int h = 0; h < 2; ++h) {
                                next[cell].f[h].assign(tmp[h].begin(), tmp[h].begin() + static_cast<int64_t>(m[h]) * nbins);
                                next[cell].n[h] = m[h];
                            }
                        }
                    }
                }
            }
            std::swap(cur, next);
            beam_prev = beam_cur;
            var_in = var_in + 1.0F;
        }
        std::memcpy(states_out, states.data(), states.size() * sizeof(State));
    });
}

} // extern "C"
