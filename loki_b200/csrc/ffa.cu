// FFA executor: device tables and scratch for one plan, and the level loop.
//
// Reference: FFA<float>::Impl::execute_unified (lib/ffa.cpp:242-310) and its
// CUDA twin FFACUDA (lib/ffa_cuda.cu:81-196). Differences by design: the
// coordinate tables are resolved once at creation (they depend on the plan
// only), no stream synchronisation happens between levels, and the scores
// entry point fuses the final merge level with the boxcar scorer.
#include <algorithm>
#include <memory>

#include "lk_ffa.hpp"

namespace lk {

void StageProfiler::begin(int kind, int level, uint32_t launches, uint64_t bytes,
                          cudaStream_t s) {
    if (!enabled) {
        return;
    }
    if (used == stages.size()) {
        Stage st{};
        LK_CUDA(cudaEventCreate(&st.start));
        LK_CUDA(cudaEventCreate(&st.stop));
        stages.push_back(st);
    }
    Stage& st = stages[used];
    st.kind = kind;
    st.level = level;
    st.launches = launches;
    st.bytes = bytes;
    LK_CUDA(cudaEventRecord(st.start, s));
}

void StageProfiler::end(cudaStream_t s) {
    if (!enabled) {
        return;
    }
    LK_CUDA(cudaEventRecord(stages[used].stop, s));
    ++used;
}

StageProfiler::~StageProfiler() {
    for (auto& st : stages) {
        cudaEventDestroy(st.start);
        cudaEventDestroy(st.stop);
    }
}

FFAExec::FFAExec(const Plan& p, int device, int storage, uint64_t max_batch_)
    : plan(p), device(device), max_batch(max_batch_) {
    require(max_batch >= 1 && max_batch <= 65535, "max_batch must lie in [1, 65535]");
    require(storage == LK_FP32, "only FP32 fold storage is implemented by this executor");
    require(plan.nparams <= 3, "the FFA executor supports nparams <= 3");
    require(plan.n_levels >= 2, "FFA::execute_unified: levels must be greater than or equal to 2");
    require(plan.cfg.nbins <= 0xffffffffULL, "nbins too large");
    DeviceGuard g(device);
    status.alloc(sizeof(uint32_t));
    LK_CUDA(cudaMemset(status.ptr, 0, sizeof(uint32_t)));

    const size_t elem = plan.nparams == 1 ? 8 : 16;
    coords.alloc(elem * plan.coord_size);
    resolve_coords_device(plan, coords.ptr, nullptr);
    LK_CUDA(cudaDeviceSynchronize());

    const uint32_t np = plan.nparams;
    bf = std::make_unique<BruteFoldDevice>(plan.param_grid(0, np - 1), plan.segment_lens[0],
                                           plan.cfg.nbins, plan.cfg.nsamps, plan.cfg.tsamp,
                                           plan.t_ref0(), status.as<uint32_t>());
    uint64_t inter = 0;  // largest level that is not the final one
    for (uint32_t l = 0; l + 1 < plan.n_levels; ++l) {
        inter = std::max(inter, plan.fold_size(l));
    }
    buf[0].alloc(sizeof(float) * inter * max_batch);
    buf[1].alloc(sizeof(float) * inter * max_batch);
    sp = make_score_params(plan.widths.data(), static_cast<uint32_t>(plan.widths.size()),
                           static_cast<uint32_t>(plan.cfg.nbins));
}

uint64_t FFAExec::device_bytes() const {
    return status.bytes + coords.bytes + buf[0].bytes + buf[1].bytes + bf->device_bytes() +
           scores_tmp.bytes + compact_scratch.bytes;
}

const void* FFAExec::level_coords(uint32_t l) const {
    const size_t elem = plan.nparams == 1 ? 8 : 16;
    return static_cast<const char*>(coords.ptr) + elem * plan.ncoords_offsets[l];
}

// Runs levels 0 .. last (inclusive) and returns the buffer holding `last`.
uint64_t FFAExec::coord_bytes(uint32_t l) const {
    return plan.ncoords[l] * (plan.nparams == 1 ? 8 : 16);
}

float* FFAExec::run_levels(const float* ts_e, const float* ts_v, uint32_t last,
                           float* final_out, cudaStream_t s, uint64_t nbatch) {
    require(nbatch >= 1 && nbatch <= max_batch, "nbatch must lie in [1, max_batch]");
    const bool taylor = plan.nparams > 1;
    const auto nbins = static_cast<uint32_t>(plan.cfg.nbins);
    float* in = (last == 0 && final_out != nullptr) ? final_out : buf[0].as<float>();
    // Algorithmic bytes: the series in (E and V) and the level-0 fold out;
    // each merge level reads the previous level and writes its own. A batch of
    // series is, level by level, one series with nbatch times the segments
    // (merges pair segments 2s and 2s + 1, never across two series).
    const uint64_t series_bytes = 8 * plan.cfg.nsamps * nbatch;
    bf->bind_inputs(ts_e, ts_v, s, nbatch);
    prof.begin(LK_STAGE_BRUTE_FOLD, 0, 1, series_bytes + 4 * plan.fold_size(0) * nbatch, s);
    bf->fold(in, s);
    prof.end(s);
    for (uint32_t l = 1; l <= last; ++l) {
        float* out = (l == last && final_out != nullptr) ? final_out : buf[l % 2].as<float>();
        prof.begin(LK_STAGE_MERGE, static_cast<int>(l), 1,
                   nbatch * (4 * (plan.fold_size(l - 1) + plan.fold_size(l))) + coord_bytes(l), s);
        const uint64_t n_inner = plan.param_counts[l][plan.nparams - 1];
        merge_level(in, out, level_coords(l), taylor, n_inner, plan.ncoords[l] / n_inner,
                    plan.ncoords[l - 1], plan.nsegments[l] * nbatch, nbins, s);
        prof.end(s);
        in = out;
    }
    return in;
}

void FFAExec::execute(const float* ts_e, const float* ts_v, float* fold, uint64_t fold_len,
                      cudaStream_t s, uint64_t nbatch) {
    const uint32_t L = plan.n_levels;
    require(fold_len >= plan.fold_size(L - 1) * nbatch, "fold must hold fold_size floats");
    DeviceGuard g(device);
    prof.reset();
    run_levels(ts_e, ts_v, L - 1, fold, s, nbatch);
}

void FFAExec::scores(const float* ts_e, const float* ts_v, float* d_scores, uint64_t len,
                     cudaStream_t s, uint64_t nbatch) {
    const uint32_t L = plan.n_levels;
    require(plan.nsegments[L - 1] == 1, "compute_ffa_scores: nsegments must be 1 for scores");
    require(len >= plan.ncoords[L - 1] * plan.widths.size() * nbatch,
            "scores must hold ncoords * n_widths floats");
    DeviceGuard g(device);
    if (!in_search) {
        prof.reset();
    }
    const float* in = run_levels(ts_e, ts_v, L - 2, nullptr, s, nbatch);
    const uint64_t nscores = plan.ncoords[L - 1] * plan.widths.size();
    prof.begin(LK_STAGE_MERGE_SCORE, static_cast<int>(L - 1), 1,
               nbatch * (4 * plan.fold_size(L - 2) + 4 * nscores) + coord_bytes(L - 1), s);
    const uint64_t n_inner = plan.param_counts[L - 1][plan.nparams - 1];
    merge_score_level(in, level_coords(L - 1), plan.nparams > 1, n_inner,
                      plan.ncoords[L - 1] / n_inner, plan.ncoords[L - 2],
                      static_cast<uint32_t>(plan.cfg.nbins), sp, LK_SCORE_PER_WIDTH, d_scores, s,
                      nbatch);
    prof.end(s);
}

void FFAExec::search(const float* ts_e, const float* ts_v, float snr_min, uint32_t* d_idx,
                     float* d_snr, uint64_t max_cands, uint64_t* d_count, cudaStream_t s,
                     uint64_t nbatch) {
    const uint32_t L = plan.n_levels;
    const uint64_t n = plan.ncoords[L - 1] * plan.widths.size() * nbatch;
    DeviceGuard g(device);
    if (scores_tmp.bytes < n * sizeof(float)) {
        scores_tmp.alloc(n * sizeof(float));
        compact_scratch.alloc(compact_scratch_bytes(n));
    }
    prof.reset();
    in_search = true;
    try {
        scores(ts_e, ts_v, scores_tmp.as<float>(), n, s, nbatch);
    } catch (...) {
        in_search = false;
        throw;
    }
    in_search = false;
    prof.begin(LK_STAGE_COMPACT, -1, 3, 8 * n, s);
    compact_ge(scores_tmp.as<float>(), n, snr_min, d_idx, d_snr, max_cands, d_count,
               compact_scratch.ptr, s);
    prof.end(s);
}

std::vector<lk_stage_time> FFAExec::profile(cudaStream_t s) {
    DeviceGuard g(device);
    LK_CUDA(cudaStreamSynchronize(s));
    std::vector<lk_stage_time> out;
    for (size_t i = 0; i < prof.used; ++i) {
        const auto& st = prof.stages[i];
        lk_stage_time t{};
        t.kind = st.kind;
        t.level = st.level;
        t.launches = st.launches;
        t.bytes = st.bytes;
        LK_CUDA(cudaEventElapsedTime(&t.ms, st.start, st.stop));
        out.push_back(t);
    }
    return out;
}

uint32_t FFAExec::read_status(cudaStream_t s) {
    DeviceGuard g(device);
    LK_CUDA(cudaStreamSynchronize(s));
    uint32_t st = 0;
    LK_CUDA(cudaMemcpy(&st, status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return st;
}

}  // namespace lk
