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
#include "loki/common/coord.hpp"
#include "loki/common/plans.hpp"
#include "loki/common/types.hpp"
#include "loki/detection/score.hpp"
#include "loki/psr_utils.hpp"
#include "loki/search/configs.hpp"

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

static loki::search::PulsarSearchConfig make_cfg(const lkref_cfg* c) {
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

} // extern "C"
