// The C ABI (include/loki_b200.h): argument checks, exception-to-status
// translation and the thread-local error message. No CUDA kernels here.
#include <cmath>
#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>

#include "lk_device.cuh"
#include "lk_dts.hpp"
#include "lk_ffa.hpp"
#include "lk_fourier.hpp"
#include "lk_kernels.hpp"
#include "lk_mc.hpp"
#include "lk_prune.hpp"
#include "lk_sweep.hpp"

struct lk_plan {
    lk::Plan plan;
};
struct lk_ffa {
    std::unique_ptr<lk::FFAExec> exec;
};
struct lk_mc {
    std::unique_ptr<lk::McExec> exec;
};
struct lk_prune {
    std::unique_ptr<lk::PruneExec> exec;
};
struct lk_sweep {
    std::unique_ptr<lk::FreqSweepExec> exec;
};
struct lk_dts {
    std::unique_ptr<lk::DtsExec> exec;
};
struct lk_fourier {
    std::unique_ptr<lk::FourierExec> exec;
};
struct lk_brute_fold {
    int device = 0;
    lk::DeviceBuffer status;
    std::unique_ptr<lk::BruteFoldDevice> bf;
};

namespace {

thread_local std::string g_error;

template <class F> int guarded(F&& f) {
    try {
        f();
        g_error.clear();
        return LK_OK;
    } catch (const lk::Error& e) {
        g_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_error = "host allocation failed";
        return LK_ERR_OOM;
    } catch (const std::exception& e) {
        g_error = e.what();
        return LK_ERR_INTERNAL;
    } catch (...) {
        g_error = "unknown error";
        return LK_ERR_INTERNAL;
    }
}

void need(const void* p, const char* name) {
    if (p == nullptr) {
        lk::fail(LK_ERR_INVALID_ARG, std::string(name) + " must not be NULL");
    }
}

}  // namespace

extern "C" {

const char* lk_last_error(void) { return g_error.c_str(); }

int lk_version(void) { return 100; }

int lk_plan_create(const lk_config* cfg, lk_plan** out) {
    return guarded([&] {
        need(cfg, "cfg");
        need(out, "out");
        auto p = std::make_unique<lk_plan>();
        p->plan = lk::make_plan(*cfg, /*sizes_only=*/true);
        *out = p.release();
    });
}

void lk_plan_destroy(lk_plan* plan) { delete plan; }

int lk_plan_get_info(const lk_plan* plan, lk_plan_info* out) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        const lk::Plan& p = plan->plan;
        std::memset(out, 0, sizeof(*out));
        out->nparams = p.nparams;
        out->n_levels = p.n_levels;
        out->nsamps = p.cfg.nsamps;
        out->nbins = p.cfg.nbins;
        out->tsamp = p.cfg.tsamp;
        out->bseg_brute = p.bseg_brute;
        out->bseg_ffa = p.bseg_ffa;
        out->tseg_brute = p.tseg_brute;
        out->tseg_ffa = p.tseg_ffa;
        for (uint32_t l = 0; l < p.n_levels; ++l) {
            out->segment_lens[l] = p.segment_lens[l];
            out->nsegments[l] = p.nsegments[l];
            out->tsegments[l] = p.tsegments[l];
            out->ncoords[l] = p.ncoords[l];
            out->ncoords_offsets[l] = p.ncoords_offsets[l];
            for (uint32_t i = 0; i < p.nparams; ++i) {
                out->param_counts[l][i] = p.param_counts[l][i];
                out->dparams[l][i] = p.dparams[l][i];
                out->dparams_actual[l][i] = p.dparams_actual[l][i];
            }
        }
        out->ncoords_offsets[p.n_levels] = p.ncoords_offsets[p.n_levels];
        out->buffer_size = p.buffer_size;
        out->fold_size = p.fold_size(p.n_levels - 1);
        out->brute_fold_size = p.fold_size(0);
        out->coord_size = p.coord_size;
        out->n_widths = static_cast<uint32_t>(p.widths.size());
        for (size_t i = 0; i < p.widths.size(); ++i) {
            out->widths[i] = p.widths[i];
        }
        out->snr_min = p.cfg.snr_min;
    });
}

int lk_plan_param_grid(const lk_plan* plan, uint32_t level, uint32_t iparam, double* out,
                       uint64_t n) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        const lk::Plan& p = plan->plan;
        lk::require(level < p.n_levels && iparam < p.nparams, "level/iparam out of range");
        const auto g = p.param_grid(level, iparam);
        std::memcpy(out, g.data(), sizeof(double) * std::min<uint64_t>(n, g.size()));
    });
}

int lk_plan_dparams(const lk_plan* plan, double tseg_cur, int kind, double* out) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        lk::require(kind >= 0 && kind <= 2, "kind must be 0, 1 or 2");
        const auto d = plan->plan.dparams_at(tseg_cur, kind);
        std::memcpy(out, d.data(), sizeof(double) * d.size());
    });
}

int lk_plan_resolve_coords(const lk_plan* plan, void* d_coords, uint64_t n_coords,
                           lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        need(d_coords, "d_coords");
        lk::require(n_coords >= plan->plan.coord_size, "coords must hold coord_size entries");
        lk::resolve_coords_device(plan->plan, d_coords, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_ffa_create(const lk_plan* plan, int device, int storage, lk_ffa** out) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        auto f = std::make_unique<lk_ffa>();
        f->exec = std::make_unique<lk::FFAExec>(plan->plan, device, storage);
        *out = f.release();
    });
}

void lk_ffa_destroy(lk_ffa* ffa) {
    if (ffa != nullptr) {
        try {
            lk::DeviceGuard g(ffa->exec->device);
            delete ffa;
        } catch (...) {
            delete ffa;
        }
    }
}

int lk_ffa_workspace_bytes(const lk_ffa* ffa, uint64_t* bytes) {
    return guarded([&] {
        need(ffa, "ffa");
        need(bytes, "bytes");
        *bytes = ffa->exec->device_bytes();
    });
}

int lk_ffa_execute(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, float* d_fold,
                   uint64_t fold_len, lk_stream_t stream) {
    return guarded([&] {
        need(ffa, "ffa");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_fold, "d_fold");
        ffa->exec->execute(d_ts_e, d_ts_v, d_fold, fold_len, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_ffa_scores(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, float* d_scores,
                  uint64_t scores_len, lk_stream_t stream) {
    return guarded([&] {
        need(ffa, "ffa");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_scores, "d_scores");
        ffa->exec->scores(d_ts_e, d_ts_v, d_scores, scores_len,
                          reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_ffa_search(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, float snr_min,
                  uint32_t* d_idx, float* d_snr, uint64_t max_cands, uint64_t* d_count,
                  lk_stream_t stream) {
    return guarded([&] {
        need(ffa, "ffa");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_count, "d_count");
        if (max_cands > 0) {
            need(d_idx, "d_idx");
            need(d_snr, "d_snr");
        }
        ffa->exec->search(d_ts_e, d_ts_v, snr_min, d_idx, d_snr, max_cands, d_count,
                          reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_ffa_create_batched(const lk_plan* plan, int device, int storage, uint64_t max_batch,
                          lk_ffa** out) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        auto f = std::make_unique<lk_ffa>();
        f->exec = std::make_unique<lk::FFAExec>(plan->plan, device, storage, max_batch);
        *out = f.release();
    });
}

int lk_ffa_execute_batch(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint64_t nbatch,
                         float* d_fold, uint64_t fold_len, lk_stream_t stream) {
    return guarded([&] {
        need(ffa, "ffa");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_fold, "d_fold");
        ffa->exec->execute(d_ts_e, d_ts_v, d_fold, fold_len, reinterpret_cast<cudaStream_t>(stream),
                           nbatch);
    });
}

int lk_ffa_scores_batch(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint64_t nbatch,
                        float* d_scores, uint64_t scores_len, lk_stream_t stream) {
    return guarded([&] {
        need(ffa, "ffa");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_scores, "d_scores");
        ffa->exec->scores(d_ts_e, d_ts_v, d_scores, scores_len,
                          reinterpret_cast<cudaStream_t>(stream), nbatch);
    });
}

int lk_ffa_search_batch(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint64_t nbatch,
                        float snr_min, uint32_t* d_idx, float* d_snr, uint64_t max_cands,
                        uint64_t* d_count, lk_stream_t stream) {
    return guarded([&] {
        need(ffa, "ffa");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_count, "d_count");
        if (max_cands > 0) {
            need(d_idx, "d_idx");
            need(d_snr, "d_snr");
        }
        ffa->exec->search(d_ts_e, d_ts_v, snr_min, d_idx, d_snr, max_cands, d_count,
                          reinterpret_cast<cudaStream_t>(stream), nbatch);
    });
}

int lk_ffa_set_batch_lengths(lk_ffa* ffa, const uint64_t* d_lengths) {
    return guarded([&] {
        need(ffa, "ffa");
        ffa->exec->batch_lens = d_lengths;
    });
}

int lk_ffa_status(lk_ffa* ffa, lk_stream_t stream, uint32_t* status) {
    return guarded([&] {
        need(ffa, "ffa");
        need(status, "status");
        *status = ffa->exec->read_status(reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_ffa_set_rescore_margin(lk_ffa* ffa, float margin_abs, float margin_rel) {
    return guarded([&] {
        need(ffa, "ffa");
        lk::require(std::isfinite(margin_abs) && std::isfinite(margin_rel) && margin_abs >= 0.0f &&
                        margin_rel >= 0.0f,
                    "rescore margins must be finite and >= 0");
        if (ffa->exec->mixed) {
            ffa->exec->margin_abs = margin_abs;
            ffa->exec->margin_rel = margin_rel;
        }
    });
}

int lk_ffa_get_rescore_margin(const lk_ffa* ffa, float* margin_abs, float* margin_rel) {
    return guarded([&] {
        need(ffa, "ffa");
        need(margin_abs, "margin_abs");
        need(margin_rel, "margin_rel");
        *margin_abs = ffa->exec->margin_abs;
        *margin_rel = ffa->exec->margin_rel;
    });
}

int lk_ffa_rescored_cells(lk_ffa* ffa, lk_stream_t stream, uint64_t* n_cells) {
    return guarded([&] {
        need(ffa, "ffa");
        need(n_cells, "n_cells");
        *n_cells = ffa->exec->rescored_cells(reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_sweep_create(const lk_config* base, const lk_sweep_options* opt, int device, int storage,
                    lk_sweep** out) {
    return guarded([&] {
        need(base, "base");
        need(out, "out");
        lk::SweepOptions o;
        if (opt != nullptr) {
            o.max_memory_gb = opt->max_memory_gb;
            o.octave_scale = opt->octave_scale;
            o.nbins_max = opt->nbins_max;
            o.max_passing_candidates = opt->max_passing_candidates;
            o.decode_chunk_widths = opt->decode_chunk_widths != 0;
            o.device_memory_model = opt->device_memory_model != 0;
            lk::require(opt->executor_mode >= 0 && opt->executor_mode <= 2,
                        "executor_mode must be 0 (auto), 1 (resident) or 2 (one chunk at a time)");
            o.executor_mode = opt->executor_mode;
            o.autotune = opt->autotune != 0;
            o.use_fourier = opt->use_fourier != 0;
            o.nbins_min_lossy_bf = opt->nbins_min_lossy_bf == 0 ? 64 : opt->nbins_min_lossy_bf;
            lk::require(opt->plan_sizes >= 0 && opt->plan_sizes <= 2, "plan_sizes must be 0, 1 or 2");
            o.plan_sizes = opt->plan_sizes;
        }
        lk::require(o.max_memory_gb > 0, "max_process_memory_gb must be positive");
        auto h = std::make_unique<lk_sweep>();
        h->exec = std::make_unique<lk::FreqSweepExec>(*base, o, device, storage);
        *out = h.release();
    });
}

void lk_sweep_destroy(lk_sweep* sw) { delete sw; }

int lk_sweep_set_profiling(lk_sweep* sw, int enable) {
    return guarded([&] {
        need(sw, "sw");
        sw->exec->set_profiling(enable != 0);
    });
}

int lk_sweep_get_profile(lk_sweep* sw, lk_stage_time* out, uint32_t max_out, uint32_t* n_out) {
    return guarded([&] {
        need(sw, "sw");
        need(n_out, "n_out");
        const auto st = sw->exec->profile(nullptr);
        const auto n = static_cast<uint32_t>(std::min<size_t>(st.size(), max_out));
        if (n > 0) {
            need(out, "out");
            std::copy(st.begin(), st.begin() + n, out);
        }
        *n_out = static_cast<uint32_t>(st.size());
    });
}

int lk_generate_ffa_regions(double p_min, double p_max, double tsamp, uint64_t nbins_min,
                            double eta_min, double octave_scale, uint64_t nbins_max,
                            double* rows, uint64_t cap, uint64_t* n_out) {
    return guarded([&] {
        need(n_out, "n_out");
        const auto rg = lk::generate_ffa_regions(p_min, p_max, tsamp, nbins_min, eta_min,
                                                 octave_scale, nbins_max);
        *n_out = rg.size();
        if (cap > 0) {
            need(rows, "rows");
        }
        for (size_t i = 0; i < rg.size() && i < cap; ++i) {
            rows[4 * i + 0] = rg[i].f_start;
            rows[4 * i + 1] = rg[i].f_end;
            rows[4 * i + 2] = static_cast<double>(rg[i].nbins);
            rows[4 * i + 3] = rg[i].eta;
        }
    });
}

int lk_sweep_nchunks(const lk_sweep* sw, uint64_t* n) {
    return guarded([&] {
        need(sw, "sw");
        need(n, "n");
        *n = sw->exec->chunks().size();
    });
}

int lk_sweep_chunk_info(const lk_sweep* sw, uint64_t i, lk_sweep_chunk* out) {
    return guarded([&] {
        need(sw, "sw");
        need(out, "out");
        const auto& ch = sw->exec->chunks();
        lk::require(i < ch.size(), "chunk index out of range");
        const auto& c = ch[i];
        const uint32_t np = c.cfg.nparams;
        out->f_min = c.cfg.param_limits[2 * (np - 1)];
        out->f_max = c.cfg.param_limits[2 * (np - 1) + 1];
        out->nominal_f_start = c.nominal_f_start;
        out->nominal_f_end = c.nominal_f_end;
        out->nbins = c.cfg.nbins;
        out->eta = c.cfg.eta;
        out->buffer_size = c.buffer_size;
        out->coord_size = c.coord_size;
        out->ncoords = c.ncoords;
        out->n_levels = c.n_levels;
        out->memory_gb = c.memory_gb;
        out->allocated_gb = c.allocated_gb;
    });
}

int lk_sweep_execute(lk_sweep* sw, const float* d_ts_e, const float* d_ts_v, lk_stream_t stream) {
    return guarded([&] {
        need(sw, "sw");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        sw->exec->execute(d_ts_e, d_ts_v, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_sweep_results(const lk_sweep* sw, double* params, float* scores, uint64_t max_out,
                     uint64_t* n_out, uint64_t* region_counts) {
    return guarded([&] {
        need(sw, "sw");
        need(n_out, "n_out");
        const auto& sc = sw->exec->scores();
        const auto& pr = sw->exec->params();
        const uint64_t n = sc.size();
        const uint64_t k = std::min(n, max_out);
        const uint64_t stride = sw->exec->nparams() + 1;
        *n_out = n;
        if (k > 0) {
            need(params, "params");
            need(scores, "scores");
            std::copy_n(pr.begin(), k * stride, params);
            std::copy_n(sc.begin(), k, scores);
        }
        if (region_counts != nullptr) {
            const auto& rc = sw->exec->region_counts();
            std::copy(rc.begin(), rc.end(), region_counts);
        }
    });
}

int lk_ffa_autotune(lk_ffa* ffa, const float* d_ts_e, const float* d_ts_v, uint32_t reps,
                    lk_tuning* out, lk_stream_t stream) {
    return guarded([&] {
        need(ffa, "ffa");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        const lk_tuning t =
            ffa->exec->autotune(d_ts_e, d_ts_v, reps, reinterpret_cast<cudaStream_t>(stream));
        if (out != nullptr) {
            *out = t;
        }
    });
}

int lk_ffa_get_tuning(const lk_ffa* ffa, lk_tuning* out) {
    return guarded([&] {
        need(ffa, "ffa");
        need(out, "out");
        lk_tuning t = ffa->exec->tuning;
        t.bf_rows = ffa->exec->bf->rows();
        t.bf_warps = ffa->exec->bf->warps();
        t.bf_stages = ffa->exec->bf->stages();
        t.bf_tmem_warps = ffa->exec->bf->tmem_warps();
        t.merge_rows_in_flight = ffa->exec->merge_pb;
        t.score_cells_per_block = ffa->exec->score_cells;
        *out = t;
    });
}

int lk_ffa_set_tuning(lk_ffa* ffa, const lk_tuning* tuning) {
    return guarded([&] {
        need(ffa, "ffa");
        need(tuning, "tuning");
        ffa->exec->apply_tuning(*tuning);
    });
}

int lk_ffa_set_profiling(lk_ffa* ffa, int enable) {
    return guarded([&] {
        need(ffa, "ffa");
        ffa->exec->prof.enabled = enable != 0;
        ffa->exec->prof.reset();
    });
}

int lk_ffa_get_profile(lk_ffa* ffa, lk_stream_t stream, lk_stage_time* out, uint32_t max_out,
                       uint32_t* n_out) {
    return guarded([&] {
        need(ffa, "ffa");
        need(n_out, "n_out");
        const auto st = ffa->exec->profile(reinterpret_cast<cudaStream_t>(stream));
        const auto n = static_cast<uint32_t>(std::min<size_t>(st.size(), max_out));
        if (n > 0) {
            need(out, "out");
            std::copy(st.begin(), st.begin() + n, out);
        }
        *n_out = static_cast<uint32_t>(st.size());
    });
}

int lk_fourier_brute_fold(const float* d_ts_e, const float* d_ts_v, uint64_t nsamps,
                          const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                          uint64_t nbins, double tsamp, double t_ref, float* d_fold,
                          uint64_t fold_len, int device, lk_stream_t stream) {
    return guarded([&] {
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(freqs, "freqs");
        need(d_fold, "d_fold");
        lk::require(nfreqs >= 1 && nfreqs <= 0xffffffffULL, "nfreqs out of range");
        lk::require(segment_len >= 1 && segment_len <= nsamps, "segment_len must lie in [1, nsamps]");
        lk::require(nbins >= 2 && nbins <= 2048, "nbins must lie in [2, 2048]");
        lk::require(reinterpret_cast<uintptr_t>(d_fold) % 8 == 0, "d_fold must be 8-byte aligned");
        const uint64_t nseg = nsamps / segment_len;
        lk::require(fold_len >= nseg * nfreqs * 2 * (nbins / 2 + 1),
                    "fold must hold nseg * nfreqs * 2 * (nbins / 2 + 1) complex values");
        lk::DeviceGuard g(device);
        const auto s = reinterpret_cast<cudaStream_t>(stream);
        lk::DeviceBuffer f(sizeof(double) * nfreqs);
        LK_CUDA(cudaMemcpyAsync(f.ptr, freqs, sizeof(double) * nfreqs, cudaMemcpyHostToDevice, s));
        lk::fourier_dft_fold(d_ts_e, d_ts_v, f.as<double>(), static_cast<uint32_t>(nfreqs),
                             segment_len, nseg, static_cast<uint32_t>(nbins), tsamp, t_ref,
                             reinterpret_cast<float2*>(d_fold), s);
        // the frequency table is freed on return: finish the launch first
        LK_CUDA(cudaStreamSynchronize(s));
    });
}

int lk_fourier_create(const lk_plan* plan, int device, uint64_t nbins_min_lossy_bf,
                      lk_fourier** out) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        auto f = std::make_unique<lk_fourier>();
        f->exec = std::make_unique<lk::FourierExec>(plan->plan, device, nbins_min_lossy_bf);
        *out = f.release();
    });
}

void lk_fourier_destroy(lk_fourier* f) {
    if (f != nullptr) {
        try {
            lk::DeviceGuard g(f->exec->device);
            delete f;
        } catch (...) {
            delete f;
        }
    }
}

int lk_fourier_info(const lk_fourier* f, uint64_t* nbins_f, uint64_t* fold_size,
                    uint64_t* fold_size_time, int* lossy, uint64_t* workspace_bytes) {
    return guarded([&] {
        need(f, "f");
        const auto& e = *f->exec;
        const uint32_t L = e.plan.n_levels;
        if (nbins_f != nullptr) {
            *nbins_f = e.nbf;
        }
        if (fold_size != nullptr) {
            *fold_size = e.fold_size(L - 1);
        }
        if (fold_size_time != nullptr) {
            *fold_size_time = e.fold_size_time(L - 1);
        }
        if (lossy != nullptr) {
            *lossy = e.lossy ? 1 : 0;
        }
        if (workspace_bytes != nullptr) {
            *workspace_bytes = e.device_bytes();
        }
    });
}

int lk_fourier_execute(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float* d_fold,
                       uint64_t fold_len, lk_stream_t stream) {
    return guarded([&] {
        need(f, "f");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_fold, "d_fold");
        lk::require(reinterpret_cast<uintptr_t>(d_fold) % 8 == 0, "d_fold must be 8-byte aligned");
        f->exec->execute(d_ts_e, d_ts_v, reinterpret_cast<float2*>(d_fold), fold_len,
                         reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_fourier_execute_time(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float* d_fold,
                            uint64_t fold_len, lk_stream_t stream) {
    return guarded([&] {
        need(f, "f");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_fold, "d_fold");
        f->exec->execute_time(d_ts_e, d_ts_v, d_fold, fold_len,
                              reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_fourier_scores(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float* d_scores,
                      uint64_t scores_len, lk_stream_t stream) {
    return guarded([&] {
        need(f, "f");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_scores, "d_scores");
        f->exec->scores(d_ts_e, d_ts_v, d_scores, scores_len,
                        reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_fourier_search(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, float snr_min,
                      uint32_t* d_idx, float* d_snr, uint64_t max_cands, uint64_t* d_count,
                      lk_stream_t stream) {
    return guarded([&] {
        need(f, "f");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_count, "d_count");
        if (max_cands > 0) {
            need(d_idx, "d_idx");
            need(d_snr, "d_snr");
        }
        f->exec->search(d_ts_e, d_ts_v, snr_min, d_idx, d_snr, max_cands, d_count,
                        reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_fourier_set_level0(lk_fourier* f, int mode) {
    return guarded([&] {
        need(f, "f");
        f->exec->set_level0(mode);
    });
}

int lk_fourier_get_level0(const lk_fourier* f, int* mode) {
    return guarded([&] {
        need(f, "f");
        need(mode, "mode");
        const auto& e = *f->exec;
        *mode = e.lossy ? LK_FOURIER_L0_AUTO
                        : (e.uses_mma() ? LK_FOURIER_L0_TENSOR_CORES : LK_FOURIER_L0_CUDA_CORES);
    });
}

int lk_fourier_autotune(lk_fourier* f, const float* d_ts_e, const float* d_ts_v, uint32_t reps,
                        float* level0_ms, lk_stream_t stream) {
    return guarded([&] {
        need(f, "f");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        const float ms = f->exec->tune_level0(d_ts_e, d_ts_v, reps, reinterpret_cast<cudaStream_t>(stream));
        if (level0_ms != nullptr) {
            *level0_ms = ms;
        }
    });
}

int lk_fourier_status(lk_fourier* f, lk_stream_t stream, uint32_t* status) {
    return guarded([&] {
        need(f, "f");
        need(status, "status");
        *status = f->exec->read_status(reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_fourier_set_profiling(lk_fourier* f, int enable) {
    return guarded([&] {
        need(f, "f");
        f->exec->prof.enabled = enable != 0;
        f->exec->prof.reset();
    });
}

int lk_fourier_get_profile(lk_fourier* f, lk_stream_t stream, lk_stage_time* out,
                           uint32_t max_out, uint32_t* n_out) {
    return guarded([&] {
        need(f, "f");
        need(n_out, "n_out");
        const auto st = f->exec->profile(reinterpret_cast<cudaStream_t>(stream));
        const auto n = static_cast<uint32_t>(std::min<size_t>(st.size(), max_out));
        if (n > 0) {
            need(out, "out");
            std::copy(st.begin(), st.begin() + n, out);
        }
        *n_out = static_cast<uint32_t>(st.size());
    });
}

int lk_brute_fold_create(const double* freqs, uint64_t nfreqs, uint64_t segment_len,
                         uint64_t nbins, uint64_t nsamps, double tsamp, double t_ref, int device,
                         lk_brute_fold** out) {
    return guarded([&] {
        need(freqs, "freqs");
        need(out, "out");
        lk::DeviceGuard g(device);
        auto b = std::make_unique<lk_brute_fold>();
        b->device = device;
        b->status.alloc(sizeof(uint32_t));
        LK_CUDA(cudaMemset(b->status.ptr, 0, sizeof(uint32_t)));
        b->bf = std::make_unique<lk::BruteFoldDevice>(std::vector<double>(freqs, freqs + nfreqs),
                                                      segment_len, nbins, nsamps, tsamp, t_ref,
                                                      b->status.as<uint32_t>());
        *out = b.release();
    });
}

void lk_brute_fold_destroy(lk_brute_fold* bf) {
    if (bf != nullptr) {
        try {
            lk::DeviceGuard g(bf->device);
            delete bf;
        } catch (...) {
            delete bf;
        }
    }
}

int lk_brute_fold_execute(lk_brute_fold* bf, const float* d_ts_e, const float* d_ts_v,
                          float* d_fold, lk_stream_t stream) {
    return guarded([&] {
        need(bf, "bf");
        need(d_ts_e, "d_ts_e");
        need(d_ts_v, "d_ts_v");
        need(d_fold, "d_fold");
        lk::DeviceGuard g(bf->device);
        bf->bf->execute(d_ts_e, d_ts_v, d_fold, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_box_width_trials(uint64_t nbins, double ducy_max, double wtsp, uint32_t* out,
                        uint32_t max_out, uint32_t* n_out) {
    return guarded([&] {
        need(out, "out");
        need(n_out, "n_out");
        const auto w = lk::box_width_trials(nbins, ducy_max, wtsp);
        lk::require(w.size() <= max_out, "output too small for the width trials");
        std::copy(w.begin(), w.end(), out);
        *n_out = static_cast<uint32_t>(w.size());
    });
}

int lk_snr_boxcar_3d(const float* d_folds, uint64_t nprofiles, uint32_t nbins,
                     const uint32_t* widths, uint32_t nwidths, int mode, float* d_scores,
                     lk_stream_t stream) {
    return guarded([&] {
        need(widths, "widths");
        lk::require(mode == LK_SCORE_PER_WIDTH || mode == LK_SCORE_MAX, "bad score mode");
        if (nprofiles == 0) {
            return;
        }
        need(d_folds, "d_folds");
        need(d_scores, "d_scores");
        const auto sp = lk::make_score_params(widths, nwidths, nbins);
        lk::score_folds(d_folds, nprofiles, nbins, true, 1.0f, sp, mode, d_scores,
                        reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_snr_boxcar_2d_max(const float* d_folds, uint64_t nprofiles, uint32_t nbins,
                         const uint32_t* widths, uint32_t nwidths, float stdnoise,
                         float* d_scores, lk_stream_t stream) {
    return guarded([&] {
        need(widths, "widths");
        if (nprofiles == 0) {
            return;
        }
        need(d_folds, "d_folds");
        need(d_scores, "d_scores");
        const auto sp = lk::make_score_params(widths, nwidths, nbins);
        // snr_boxcar_impl<false, ...>: inv_stdnoise = 1.0F / stdnoise (lib/score.cpp:117).
        const float inv = 1.0f / stdnoise;
        lk::score_folds(d_folds, nprofiles, nbins, false, inv, sp, LK_SCORE_MAX, d_scores,
                        reinterpret_cast<cudaStream_t>(stream));
    });
}

uint64_t lk_compact_scratch_bytes(uint64_t n) { return lk::compact_scratch_bytes(n); }

int lk_compact_ge(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx, float* d_vals,
                  uint64_t max_out, uint64_t* d_count, void* d_scratch, lk_stream_t stream) {
    return guarded([&] {
        need(d_count, "d_count");
        if (n > 0) {
            need(d_scores, "d_scores");
            need(d_scratch, "d_scratch");
        }
        if (max_out > 0) {
            need(d_idx, "d_idx");
            need(d_vals, "d_vals");
        }
        lk::compact_ge(d_scores, n, thr, d_idx, d_vals, max_out, d_count, d_scratch,
                       reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_dts_create(const lk_dts_config* cfg, int device, lk_dts** out) {
    return guarded([&] {
        need(cfg, "cfg");
        need(out, "out");
        auto d = std::make_unique<lk_dts>();
        d->exec = std::make_unique<lk::DtsExec>(*cfg, device);
        *out = d.release();
    });
}

void lk_dts_destroy(lk_dts* dts) { delete dts; }

int lk_dts_run(lk_dts* dts, uint32_t thres_neigh, lk_stream_t stream) {
    return guarded([&] {
        need(dts, "dts");
        dts->exec->run(thres_neigh, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_dts_info(const lk_dts* dts, uint32_t* nstages, uint32_t* nthresholds, uint32_t* nprobs,
                uint32_t* nbins, uint32_t* nwidths) {
    return guarded([&] {
        need(dts, "dts");
        const lk::DtsExec& e = *dts->exec;
        if (nstages) *nstages = e.nstages();
        if (nthresholds) *nthresholds = e.nthresholds();
        if (nprobs) *nprobs = e.nprobs();
        if (nbins) *nbins = e.nbins();
        if (nwidths) *nwidths = static_cast<uint32_t>(e.m_widths.size());
    });
}

int lk_dts_arrays(const lk_dts* dts, float* profile, float* thresholds, float* probs,
                  float* guess_path, uint32_t* widths) {
    return guarded([&] {
        need(dts, "dts");
        const lk::DtsExec& e = *dts->exec;
        if (profile) std::copy(e.m_profile.begin(), e.m_profile.end(), profile);
        if (thresholds) std::copy(e.m_thresholds.begin(), e.m_thresholds.end(), thresholds);
        if (probs) std::copy(e.m_probs.begin(), e.m_probs.end(), probs);
        if (guess_path) std::copy(e.m_guess.begin(), e.m_guess.end(), guess_path);
        if (widths) std::copy(e.m_widths.begin(), e.m_widths.end(), widths);
    });
}

int lk_dts_transitions(const lk_dts* dts, uint64_t* n) {
    return guarded([&] {
        need(dts, "dts");
        need(n, "n");
        *n = dts->exec->m_transitions;
    });
}

int lk_dts_states(const lk_dts* dts, lk_dts_state* out, uint64_t n) {
    return guarded([&] {
        need(dts, "dts");
        need(out, "out");
        const auto& st = dts->exec->m_states;
        lk::require(!st.empty(), "run the scheme before reading its states");
        lk::require(n >= st.size(), "out must hold nstages * nthresholds * nprobs states");
        std::copy(st.begin(), st.end(), out);
    });
}

int lk_dts_best_path(const lk_dts* dts, float min_pd, float* out, uint32_t* n) {
    return guarded([&] {
        need(dts, "dts");
        need(out, "out");
        need(n, "n");
        const std::vector<float> p = dts->exec->best_path(min_pd);
        std::copy(p.begin(), p.end(), out);
        *n = static_cast<uint32_t>(p.size());
    });
}

int lk_dts_plan(const lk_dts_config* cfg, float* profile, float* thresholds, float* probs,
                float* guess_path, uint32_t* widths, uint32_t* nwidths) {
    return guarded([&] {
        need(cfg, "cfg");
        need(cfg->branching_pattern, "branching_pattern");
        lk::require(cfg->nstages >= 1 && cfg->nthresholds >= 2 && cfg->nprobs >= 2 && cfg->nbins >= 4,
                    "invalid scheme configuration");
        const std::vector<float> bp(cfg->branching_pattern, cfg->branching_pattern + cfg->nstages);
        if (profile) {
            const auto v = lk::dts_profile(cfg->nbins, cfg->ref_ducy, 0.5F);
            std::copy(v.begin(), v.end(), profile);
        }
        if (thresholds) {
            const auto v = lk::dts_thresholds(0.1F, cfg->snr_final, cfg->nthresholds);
            std::copy(v.begin(), v.end(), thresholds);
        }
        if (probs) {
            const auto v = lk::dts_probs(cfg->nprobs, cfg->prob_min);
            std::copy(v.begin(), v.end(), probs);
        }
        if (guess_path) {
            const auto v = lk::dts_guess_scheme(cfg->nstages, cfg->snr_final, bp, cfg->trials_start, 1E10F);
            std::copy(v.begin(), v.end(), guess_path);
        }
        const auto w = lk::box_width_trials(cfg->nbins, cfg->ducy_max, cfg->wtsp);
        if (widths) {
            lk::require(w.size() <= LK_MAX_WIDTHS, "too many widths");
            std::copy(w.begin(), w.end(), widths);
        }
        if (nwidths) {
            *nwidths = static_cast<uint32_t>(w.size());
        }
    });
}

int lk_dts_normal_lut(float* out, uint64_t n) {
    return guarded([&] {
        need(out, "out");
        lk::require(n >= lk::kDtsLutSize, "out must hold 131073 floats");
        const std::vector<float> lut = lk::normal_lut();
        std::copy(lut.begin(), lut.end(), out);
    });
}

int lk_wait_check(uint32_t limit_us, int complete, uint32_t* status, lk_stream_t stream) {
    int rc = LK_OK;
    const int g = guarded([&] {
        need(status, "status");
        lk::DeviceBuffer word(sizeof(uint32_t));
        *status = lk::wait_check(static_cast<uint64_t>(limit_us) * 1000ull, complete != 0,
                                 word.as<uint32_t>(), reinterpret_cast<cudaStream_t>(stream));
        if ((*status & lk::dev::kStatusWaitTimeout) != 0) {
            rc = LK_ERR_DEVICE_TIMEOUT;
        }
    });
    if (g != LK_OK) {
        return g;
    }
    if (rc != LK_OK) {
        g_error = "a bounded device-side wait gave up (status word " + std::to_string(*status) + ")";
    }
    return rc;
}

int lk_compact_ge_noalloc(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx,
                          float* d_vals, uint64_t max_out, uint64_t* d_count,
                          lk_stream_t stream) {
    return guarded([&] {
        need(d_count, "d_count");
        if (n > 0) {
            need(d_scores, "d_scores");
        }
        if (max_out > 0) {
            need(d_idx, "d_idx");
            need(d_vals, "d_vals");
        }
        lk::compact_ge_noalloc(d_scores, n, thr, d_idx, d_vals, max_out, d_count,
                               reinterpret_cast<cudaStream_t>(stream));
    });
}

// ---- pruning leaf step ------------------------------------------------------

int lk_prune_create(const lk_plan* plan, uint64_t max_sugg, uint64_t batch_size,
                    uint64_t branch_max, int conservative, int device, lk_prune** out) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        auto h = std::make_unique<lk_prune>();
        if (branch_max == 0) {
            branch_max = plan->plan.prune_branch_max(conservative != 0);
        }
        h->exec = std::make_unique<lk::PruneExec>(plan->plan, max_sugg, batch_size, branch_max,
                                                  conservative != 0, device);
        *out = h.release();
    });
}

int lk_prune_create_basis(const lk_plan* plan, uint64_t max_sugg, uint64_t batch_size,
                          uint64_t branch_max, int conservative, int poly_basis, int device,
                          lk_prune** out) {
    return guarded([&] {
        need(plan, "plan");
        need(out, "out");
        lk::require(poly_basis == LK_BASIS_TAYLOR || poly_basis == LK_BASIS_CHEBYSHEV,
                    "Unknown poly_basis. Valid options: 'taylor', 'chebyshev'");
        lk::require(!(poly_basis == LK_BASIS_CHEBYSHEV && conservative != 0),
                    "Conservative tile not implemented for Chebyshev basis");
        auto h = std::make_unique<lk_prune>();
        if (branch_max == 0) {
            branch_max = plan->plan.prune_branch_max(conservative != 0, poly_basis);
        }
        h->exec = std::make_unique<lk::PruneExec>(plan->plan, max_sugg, batch_size, branch_max,
                                                  conservative != 0, device, poly_basis);
        *out = h.release();
    });
}

int lk_plan_branching_pattern_basis(const lk_plan* plan, uint64_t ref_seg, int conservative,
                                    int poly_basis, double* out, uint64_t max_out,
                                    uint64_t* n_out) {
    return guarded([&] {
        need(plan, "plan");
        need(n_out, "n_out");
        lk::require(poly_basis == LK_BASIS_TAYLOR || poly_basis == LK_BASIS_CHEBYSHEV,
                    "Invalid poly_basis for branching pattern generation");
        if (poly_basis == LK_BASIS_CHEBYSHEV) {
            lk::require(conservative == 0,
                        "Conservative tile is not supported for chebyshev branching pattern "
                        "generation");
        }
        const auto bp = poly_basis == LK_BASIS_CHEBYSHEV
                            ? plan->plan.branching_pattern_cheby(ref_seg)
                            : plan->plan.branching_pattern(ref_seg, conservative != 0);
        *n_out = bp.size();
        if (max_out > 0) {
            need(out, "out");
        }
        std::copy_n(bp.begin(), std::min<uint64_t>(bp.size(), max_out), out);
    });
}

void lk_prune_destroy(lk_prune* pr) { delete pr; }

int lk_plan_branching_pattern(const lk_plan* plan, uint64_t ref_seg, int conservative,
                              double* out, uint64_t max_out, uint64_t* n_out) {
    return guarded([&] {
        need(plan, "plan");
        need(n_out, "n_out");
        const auto bp = plan->plan.branching_pattern(ref_seg, conservative != 0);
        *n_out = bp.size();
        if (max_out > 0) {
            need(out, "out");
        }
        std::copy_n(bp.begin(), std::min<uint64_t>(bp.size(), max_out), out);
    });
}

int lk_prune_run_many(lk_prune* const* prs, uint64_t n, const float* d_ffa_fold,
                      const uint64_t* ref_segs, const float* thresholds, uint64_t n_thresholds,
                      uint64_t n_iters, lk_prune_stats* stats, uint64_t max_stats, uint64_t* n_stats,
                      lk_stream_t stream) {
    return guarded([&] {
        need(prs, "prs");
        need(ref_segs, "ref_segs");
        need(d_ffa_fold, "d_ffa_fold");
        need(n_stats, "n_stats");
        lk::require(n >= 1, "n must be positive");
        if (n_thresholds > 0) {
            need(thresholds, "thresholds");
        }
        if (max_stats > 0) {
            need(stats, "stats");
        }
        std::vector<lk::PruneExec*> ex(n);
        for (uint64_t k = 0; k < n; ++k) {
            need(prs[k], "prs[k]");
            ex[k] = prs[k]->exec.get();
        }
        const auto out = lk::PruneExec::run_many(ex, d_ffa_fold, std::vector<uint64_t>(ref_segs, ref_segs + n),
                                                 thresholds, n_thresholds, n_iters,
                                                 reinterpret_cast<cudaStream_t>(stream));
        for (uint64_t k = 0; k < n; ++k) {
            n_stats[k] = out[k].size();
            std::copy_n(out[k].begin(), std::min<uint64_t>(out[k].size(), max_stats), stats + k * max_stats);
        }
    });
}

int lk_prune_set_tail(lk_prune* pr, int enable) {
    return guarded([&] {
        need(pr, "pr");
        pr->exec->tail_enabled = enable != 0;
    });
}

int lk_prune_run(lk_prune* pr, const float* d_ffa_fold, uint64_t ref_seg,
                 const float* thresholds, uint64_t n_thresholds, uint64_t n_iters,
                 lk_prune_stats* stats, uint64_t max_stats, uint64_t* n_stats,
                 lk_stream_t stream) {
    return guarded([&] {
        need(pr, "pr");
        need(d_ffa_fold, "d_ffa_fold");
        need(n_stats, "n_stats");
        if (n_thresholds > 0) {
            need(thresholds, "thresholds");
        }
        const auto st = pr->exec->run(d_ffa_fold, ref_seg, thresholds, n_thresholds, n_iters,
                                      reinterpret_cast<cudaStream_t>(stream));
        *n_stats = st.size();
        if (max_stats > 0) {
            need(stats, "stats");
        }
        std::copy_n(st.begin(), std::min<uint64_t>(st.size(), max_stats), stats);
    });
}

int lk_prune_finalize(lk_prune* pr, const float* d_ffa_fold, lk_stream_t stream) {
    return guarded([&] {
        need(pr, "pr");
        need(d_ffa_fold, "d_ffa_fold");
        pr->exec->finalize(d_ffa_fold, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_prune_get_scores_ep(const lk_prune* pr, float* d_scores_ep, uint64_t max_out,
                           lk_stream_t stream) {
    return guarded([&] {
        need(pr, "pr");
        lk::require(pr->exec->tree_size() <= max_out, "max_out is smaller than the tree size");
        pr->exec->copy_scores_ep(d_scores_ep, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_prune_tree_size(const lk_prune* pr, uint64_t* n) {
    return guarded([&] {
        need(pr, "pr");
        need(n, "n");
        *n = pr->exec->tree_size();
    });
}

int lk_prune_get_tree(const lk_prune* pr, double* d_leaves, float* d_folds, float* d_scores,
                      uint64_t max_out, lk_stream_t stream) {
    return guarded([&] {
        need(pr, "pr");
        lk::require(pr->exec->tree_size() <= max_out, "max_out is smaller than the tree size");
        pr->exec->copy_tree(d_leaves, d_folds, d_scores, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_taylor_seed(const lk_plan* plan, double* d_leaves, lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        need(d_leaves, "d_leaves");
        lk::taylor_seed(plan->plan, d_leaves, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_taylor_branch(const lk_plan* plan, const double* d_leaves, uint64_t n, double scale_cur,
                     uint64_t branch_max, double* d_out, uint32_t* d_origins, uint64_t max_out,
                     uint64_t* n_out, lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        need(n_out, "n_out");
        if (n > 0) {
            need(d_leaves, "d_leaves");
        }
        if (max_out > 0) {
            need(d_out, "d_out");
            need(d_origins, "d_origins");
        }
        *n_out = lk::taylor_branch(plan->plan, d_leaves, n, scale_cur, branch_max, d_out,
                                   d_origins, max_out, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_taylor_resolve(const lk_plan* plan, const double* d_leaves, uint64_t n,
                      const double* coords, uint32_t* d_param_idx, float* d_phase_shift,
                      lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        need(coords, "coords");
        if (n > 0) {
            need(d_leaves, "d_leaves");
            need(d_param_idx, "d_param_idx");
            need(d_phase_shift, "d_phase_shift");
        }
        lk::taylor_resolve(plan->plan, d_leaves, n, coords, d_param_idx, d_phase_shift,
                           reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_taylor_transform(const lk_plan* plan, double* d_leaves, uint64_t n_leaves,
                        const uint32_t* d_indices, uint64_t n, double t_next, double t_cur,
                        int conservative, lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        if (n > 0) {
            need(d_leaves, "d_leaves");
            need(d_indices, "d_indices");
        }
        lk::taylor_transform(plan->plan, d_leaves, n_leaves, d_indices, n, t_next, t_cur,
                             conservative != 0, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_taylor_to_cheby(double* d_leaves, uint64_t n, uint32_t nparams, double ts,
                       lk_stream_t stream) {
    return guarded([&] {
        if (n > 0) {
            need(d_leaves, "d_leaves");
        }
        lk::basis_convert(d_leaves, n, nparams, ts, true, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_cheby_to_taylor(double* d_leaves, uint64_t n, uint32_t nparams, double ts,
                       lk_stream_t stream) {
    return guarded([&] {
        if (n > 0) {
            need(d_leaves, "d_leaves");
        }
        lk::basis_convert(d_leaves, n, nparams, ts, false, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_cheby_branch(const lk_plan* plan, double* d_leaves, uint64_t n, double t_cur, double s_cur,
                    double t_prev, double s_prev, uint64_t branch_max, double* d_out,
                    uint32_t* d_origins, uint64_t max_out, uint64_t* n_out, lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        need(n_out, "n_out");
        if (n > 0) {
            need(d_leaves, "d_leaves");
        }
        if (max_out > 0) {
            need(d_out, "d_out");
            need(d_origins, "d_origins");
        }
        *n_out = lk::cheby_branch(plan->plan, d_leaves, n, t_cur, s_cur, t_prev, s_prev,
                                  branch_max, d_out, d_origins, max_out,
                                  reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_cheby_resolve(const lk_plan* plan, const double* d_leaves, uint64_t n,
                     const double* coords, uint32_t* d_param_idx, float* d_phase_shift,
                     lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        need(coords, "coords");
        if (n > 0) {
            need(d_leaves, "d_leaves");
            need(d_param_idx, "d_param_idx");
            need(d_phase_shift, "d_phase_shift");
        }
        lk::cheby_resolve(plan->plan, d_leaves, n, coords, d_param_idx, d_phase_shift,
                          reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_cheby_transform(const lk_plan* plan, double* d_leaves, uint64_t n_leaves,
                       const uint32_t* d_indices, uint64_t n, double t_next, double s_next,
                       double t_cur, double s_cur, lk_stream_t stream) {
    return guarded([&] {
        need(plan, "plan");
        if (n > 0) {
            need(d_leaves, "d_leaves");
            need(d_indices, "d_indices");
        }
        lk::cheby_transform(plan->plan, d_leaves, n_leaves, d_indices, n, t_next, s_next, t_cur,
                            s_cur, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_shift_add_batch(const float* d_folds_tree, const uint32_t* d_indices_tree,
                       const float* d_folds_ffa, uint64_t n_ffa, const uint32_t* d_indices_ffa,
                       const float* d_phase_shift, float* d_folds_out, uint32_t nbins,
                       uint64_t n, uint64_t physical_start, uint64_t capacity,
                       lk_stream_t stream) {
    return guarded([&] {
        if (n > 0) {
            need(d_folds_tree, "d_folds_tree");
            need(d_indices_tree, "d_indices_tree");
            need(d_folds_ffa, "d_folds_ffa");
            need(d_indices_ffa, "d_indices_ffa");
            need(d_phase_shift, "d_phase_shift");
            need(d_folds_out, "d_folds_out");
        }
        lk::shift_add_batch(d_folds_tree, d_indices_tree, d_folds_ffa, n_ffa, d_indices_ffa,
                            d_phase_shift, d_folds_out, nbins, n, physical_start, capacity,
                            reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_score_filter(const float* d_folds, uint64_t n, uint32_t nbins, const uint32_t* widths,
                    uint32_t nwidths, float threshold, float* d_scores, uint32_t* d_indices,
                    uint64_t* d_count, lk_stream_t stream) {
    return guarded([&] {
        need(widths, "widths");
        need(d_count, "d_count");
        const auto s = reinterpret_cast<cudaStream_t>(stream);
        const auto sp = lk::make_score_params(widths, nwidths, nbins);
        if (n == 0) {
            LK_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), s));
            return;
        }
        need(d_folds, "d_folds");
        need(d_scores, "d_scores");
        need(d_indices, "d_indices");
        lk::score_folds(d_folds, n, nbins, true, 1.0f, sp, LK_SCORE_MAX, d_scores, s);
        lk::DeviceBuffer scratch(lk::compact_scratch_bytes(n));
        lk::DeviceBuffer vals(n * sizeof(float));
        lk::compact_ge(d_scores, n, threshold, d_indices, vals.as<float>(), n, d_count,
                       scratch.ptr, s);
        LK_CUDA(cudaStreamSynchronize(s));
    });
}

// ---- Monte-Carlo threshold stage ----------------------------------------------

int lk_mc_create(uint64_t max_trials, uint32_t nbins, const uint32_t* widths, uint32_t nwidths,
                 int device, lk_mc** out) {
    return guarded([&] {
        need(widths, "widths");
        need(out, "out");
        auto h = std::make_unique<lk_mc>();
        h->exec = std::make_unique<lk::McExec>(max_trials, nbins, widths, nwidths, device);
        *out = h.release();
    });
}

void lk_mc_destroy(lk_mc* mc) { delete mc; }

int lk_mc_stage(lk_mc* mc, const float* d_folds_in, uint64_t ntrials_in, const uint32_t* d_src,
                uint64_t ntrials, const float* d_noise, uint64_t nrows, const float* d_signal,
                int signal_per_trial,
                float signal_scale, const uint32_t* d_rowmap, float var_in, float var_add,
                float threshold, const float* thresholds, uint32_t n_thr,
                const uint8_t* d_class, float* d_folds_out, uint32_t* d_ids_out,
                uint64_t* d_count, uint64_t* d_counts, float* d_max_snr, lk_stream_t stream) {
    return guarded([&] {
        need(mc, "mc");
        need(d_count, "d_count");
        if (ntrials > 0) {
            need(d_folds_in, "d_folds_in");
            need(d_noise, "d_noise");
            need(d_signal, "d_signal");
            need(d_folds_out, "d_folds_out");
        }
        if (n_thr > 0) {
            need(d_counts, "d_counts");
        }
        lk::McStage st;
        st.d_folds_in = d_folds_in;
        st.ntrials_in = ntrials_in;
        st.d_src = d_src;
        st.ntrials = ntrials;
        st.d_noise = d_noise;
        st.nrows = nrows;
        st.d_signal = d_signal;
        st.signal_per_trial = signal_per_trial != 0;
        st.signal_scale = signal_scale;
        st.d_rowmap = d_rowmap;
        st.var_in = var_in;
        st.var_add = var_add;
        st.threshold = threshold;
        st.thresholds = thresholds;
        st.n_thr = n_thr;
        st.d_class = d_class;
        st.d_folds_out = d_folds_out;
        st.d_ids_out = d_ids_out;
        st.d_count = d_count;
        st.d_counts = d_counts;
        st.d_max_snr = d_max_snr;
        mc->exec->stage(st, reinterpret_cast<cudaStream_t>(stream));
    });
}

int lk_mc_status(lk_mc* mc, lk_stream_t stream, uint32_t* status) {
    return guarded([&] {
        need(mc, "mc");
        need(status, "status");
        *status = mc->exec->read_status(reinterpret_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"
