// Test and benchmark infrastructure only: a C ABI over the reference's own
// GPU FFA (algorithms::FFACUDA<float> and FFACUDA<ComplexTypeCUDA>,
// lib/ffa_cuda.cu) and its GPU boxcar scorer (detection::snr_boxcar_3d_cuda_d,
// lib/score_cuda.cu), compiled from the reference checkout's lib/*_cuda.cu by
// oracle/Makefile (target refgpu). bench.py times the reference's GPU path with
// it beside this library's; the product never links it.
#include <cuda_runtime.h>

#include <cstdint>
#include <exception>
#include <memory>
#include <optional>
#include <span>
#include <string>
#include <vector>

#include <cuda/std/span>
#include <spdlog/spdlog.h>

#include "loki/algorithms/ffa.hpp"
#include "loki/common/types.hpp"
#include "loki/detection/score.hpp"
#include "loki/search/configs.hpp"

namespace {

thread_local std::string g_last_error;

template <class F> int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return 1;
    } catch (...) {
        g_last_error = "unknown exception";
        return 1;
    }
}

struct QuietLogs {
    QuietLogs() { spdlog::set_level(spdlog::level::warn); }
};
const QuietLogs g_quiet_logs;

}  // namespace

extern "C" {

// The same plain-C configuration as oracle/ref_capi.cpp's lkref_cfg.
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

struct lkrefg_ffa {
    std::unique_ptr<loki::search::PulsarSearchConfig> cfg;
    std::unique_ptr<loki::algorithms::FFACUDA<float>> time;
    std::unique_ptr<loki::algorithms::FFACUDA<loki::ComplexTypeCUDA>> fourier;
    uint64_t fold_len = 0;        // floats the execute call wants
    uint64_t fold_size_time = 0;  // floats of the final fold in time
    uint64_t ncoords_final = 0;
};

const char* lkrefg_last_error(void) { return g_last_error.c_str(); }

int lkrefg_create(const lkref_cfg* c, int device, int use_fourier, lkrefg_ffa** out) {
    return guarded([&] {
        std::vector<loki::ParamLimit> lims(c->nparams);
        for (uint32_t i = 0; i < c->nparams; ++i) {
            lims[i] = {.min = c->limits[2 * i], .max = c->limits[(2 * i) + 1]};
        }
        std::optional<loki::SizeType> bb, bf;
        if (c->bseg_brute != 0) {
            bb = c->bseg_brute;
        }
        if (c->bseg_ffa != 0) {
            bf = c->bseg_ffa;
        }
        auto h = std::make_unique<lkrefg_ffa>();
        h->cfg = std::make_unique<loki::search::PulsarSearchConfig>(
            c->nsamps, c->tsamp, c->nbins, c->eta, lims, c->ducy_max, c->wtsp, use_fourier != 0,
            c->nthreads, /*max_process_memory_gb=*/8.0, /*octave_scale=*/2.0, /*nbins_max=*/1024,
            /*nbins_min_lossy_bf=*/64, bb, bf);
        if (use_fourier != 0) {
            h->fourier = std::make_unique<loki::algorithms::FFACUDA<loki::ComplexTypeCUDA>>(*h->cfg, device);
            const auto& p = h->fourier->get_plan();
            h->fold_len = 2 * p.get_buffer_size();
            h->fold_size_time = p.get_fold_size_time();
            h->ncoords_final = p.get_ncoords().back();
        } else {
            h->time = std::make_unique<loki::algorithms::FFACUDA<float>>(*h->cfg, device);
            const auto& p = h->time->get_plan();
            h->fold_len = p.get_buffer_size();
            h->fold_size_time = p.get_fold_size();
            h->ncoords_final = p.get_ncoords().back();
        }
        *out = h.release();
    });
}

void lkrefg_destroy(lkrefg_ffa* h) { delete h; }

int lkrefg_info(const lkrefg_ffa* h, uint64_t* fold_len, uint64_t* fold_size_time,
                uint64_t* ncoords_final) {
    return guarded([&] {
        *fold_len = h->fold_len;
        *fold_size_time = h->fold_size_time;
        *ncoords_final = h->ncoords_final;
    });
}

// FFACUDA::execute on device spans (the final fold in time, fold_len floats
// of scratch), then snr_boxcar_3d_cuda_d of the final fold with the given
// device widths into d_scores [ncoords_final][nw], all on `stream`.
int lkrefg_scores(lkrefg_ffa* h, const float* d_e, const float* d_v, uint64_t nsamps, float* d_fold,
                  const uint32_t* d_widths, uint64_t nw, float* d_scores, void* stream) {
    return guarded([&] {
        const auto s = static_cast<cudaStream_t>(stream);
        cuda::std::span<const float> e(d_e, nsamps), v(d_v, nsamps);
        cuda::std::span<float> fold(d_fold, h->fold_len);
        if (h->fourier) {
            h->fourier->execute(e, v, fold, s);
        } else {
            h->time->execute(e, v, fold, s);
        }
        loki::detection::snr_boxcar_3d_cuda_d(
            cuda::std::span<const float>(d_fold, h->fold_size_time),
            cuda::std::span<const uint32_t>(d_widths, nw),
            cuda::std::span<float>(d_scores, h->ncoords_final * nw), h->ncoords_final,
            h->cfg->get_nbins(), s);
    });
}

}  // extern "C"
