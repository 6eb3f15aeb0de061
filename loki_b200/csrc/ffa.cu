// FFA executor: device tables and scratch for one plan, and the level loop.
//
// Reference: FFA<float>::Impl::execute_unified (lib/ffa.cpp:242-310) and its
// CUDA twin FFACUDA (lib/ffa_cuda.cu:81-196). Differences by design: the
// coordinate tables are resolved once at creation (they depend on the plan
// only), no stream synchronisation happens between levels, and the scores
// entry point fuses the final merge level with the boxcar scorer.
#include <algorithm>
#include <cmath>
#include <memory>

#include "lk_ffa.hpp"
#include "lk_score.cuh"

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
    require(!plan.offsets_overflow, "coordinate offsets exceed 32 bits");
    require(max_batch >= 1 && max_batch <= 65535, "max_batch must lie in [1, 65535]");
    require(storage == LK_FP32 || storage == LK_BF16 || storage == LK_FP16,
            "fold storage must be LK_FP32, LK_BF16 or LK_FP16");
    if (storage == LK_FP16) {
        // Level L-2 holds sums of nsamps / 2 samples per bin: its V row
        // exceeds FP16's largest finite value (65504) once nsamps / nbins
        // passes about 2^17, so FP16 without a per-level scale is unsafe.
        fail(LK_ERR_UNSUPPORTED, "FP16 fold storage is not implemented (use LK_BF16)");
    }
    mixed = storage == LK_BF16;
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
    if (!mixed) {
        uint64_t inter = 0;  // largest level that is not the final one
        for (uint32_t l = 0; l + 1 < plan.n_levels; ++l) {
            inter = std::max(inter, plan.fold_size(l));
        }
        buf[0].alloc(sizeof(float) * inter * max_batch);
        buf[1].alloc(sizeof(float) * inter * max_batch);
    } else {
        const uint32_t L = plan.n_levels;
        require(L <= kRescoreMaxLevels && plan.nsegments[0] <= kRescoreMaxLeaves,
                "BF16 storage supports at most 8192 level-0 segments");
        uint64_t inter = 1;  // largest BF16 level (1 .. L-2)
        for (uint32_t l = 1; l + 1 < L; ++l) {
            inter = std::max(inter, plan.fold_size(l));
        }
        fold0.alloc(sizeof(float) * plan.fold_size(0) * max_batch);
        buf[0].alloc(2 * inter * max_batch);  // BF16
        buf[1].alloc(2 * inter * max_batch);
        rtree.n_levels = L;
        rtree.nbins = static_cast<uint32_t>(plan.cfg.nbins);
        rtree.ncoords0 = plan.ncoords[0];
        rtree.ncoords_final = plan.ncoords[L - 1];
        rtree.fold0_size = plan.fold_size(0);
        for (uint32_t l = 1; l < L; ++l) {
            rtree.level_coords[l] = level_coords(l);
        }
        // Rounding model: each BF16 store moves a value by at most 2^-8 of
        // its magnitude (round to nearest, 8-bit significand), uniformly
        // distributed. Noise-dominated bins: the L-2 stored levels add
        // independent errors whose S/N effect has RMS 2^-8 sqrt((L-2)/3);
        // signal-dominated bins: RMS 2^-8 / sqrt(3) of the S/N. The V rows
        // are positive, so their relative error is at most (L-2) 2^-8, and
        // S/N depends on V through 1/sqrt(V). The margin takes 12 standard
        // deviations of the random parts plus the V bound.
        const double u = std::ldexp(1.0, -8);
        const double nst = static_cast<double>(L >= 2 ? L - 2 : 0);
        margin_abs = static_cast<float>(12.0 * u * std::sqrt(nst / 3.0));
        margin_rel = static_cast<float>(0.5 * nst * u + (nst > 0 ? 12.0 * u / std::sqrt(3.0) : 0.0));
    }
    sp = make_score_params(plan.widths.data(), static_cast<uint32_t>(plan.widths.size()),
                           static_cast<uint32_t>(plan.cfg.nbins));
    if (plan.nsegments[plan.n_levels - 1] == 1 &&
        make_mask_score_params(sp, static_cast<uint32_t>(plan.cfg.nbins), &mp)) {
        wm = true;
        normtab.alloc(sizeof(float) * kNormTableSize);
        norm_table_fill(normtab.as<float>(), nullptr);
        LK_CUDA(cudaDeviceSynchronize());
    }
}

uint64_t FFAExec::device_bytes() const {
    return status.bytes + coords.bytes + buf[0].bytes + buf[1].bytes + fold0.bytes +
           bf->device_bytes() + scores_tmp.bytes + compact_scratch.bytes + cmax.bytes +
           cells.bytes + cell_vals.bytes + cell_count.bytes + cell_scratch.bytes + normtab.bytes +
           blk_counts.bytes + blk_offsets.bytes;
}

float FFAExec::rescore_threshold(float snr_min) const {
    const float lo = (snr_min - margin_abs) / (1.0f + margin_rel);
    return std::nextafter(lo, -INFINITY);
}

const void* FFAExec::level_coords(uint32_t l) const {
    const size_t elem = plan.nparams == 1 ? 8 : 16;
    return static_cast<const char*>(coords.ptr) + elem * plan.ncoords_offsets[l];
}

// Runs levels 0 .. last (inclusive) and returns the buffer holding `last`.
uint64_t FFAExec::coord_bytes(uint32_t l) const {
    return plan.ncoords[l] * (plan.nparams == 1 ? 8 : 16);
}

const void* FFAExec::run_levels(const float* ts_e, const float* ts_v, uint32_t last,
                               float* final_out, cudaStream_t s, uint64_t nbatch,
                               bool* last_bf16) {
    require(nbatch >= 1 && nbatch <= max_batch, "nbatch must lie in [1, max_batch]");
    const bool taylor = plan.nparams > 1;
    const auto nbins = static_cast<uint32_t>(plan.cfg.nbins);
    // Level l is BF16 when the storage is mixed, l >= 1, and it is not the
    // caller's FP32 output.
    auto is_bf16 = [&](uint32_t l) { return mixed && l >= 1 && !(l == last && final_out); };
    auto elem = [&](uint32_t l) -> uint64_t { return is_bf16(l) ? 2 : 4; };
    void* in = (last == 0 && final_out != nullptr) ? final_out
               : mixed                             ? fold0.ptr
                                                   : buf[0].ptr;
    // Algorithmic bytes: the series in (E and V) and the level-0 fold out;
    // each merge level reads the previous level and writes its own. A batch of
    // series is, level by level, one series with nbatch times the segments
    // (merges pair segments 2s and 2s + 1, never across two series).
    const uint64_t series_bytes = 8 * plan.cfg.nsamps * nbatch;
    if (bf->interleaves()) {
        // (e, v) pairs for the packed brute fold: series in, pairs out
        prof.begin(LK_STAGE_INTERLEAVE, 0, 1, 2 * series_bytes, s);
        bf->bind_inputs(ts_e, ts_v, s, nbatch);
        prof.end(s);
    } else {
        bf->bind_inputs(ts_e, ts_v, s, nbatch);
    }
    prof.begin(LK_STAGE_BRUTE_FOLD, 0, 1, series_bytes + 4 * plan.fold_size(0) * nbatch, s);
    bf->fold(static_cast<float*>(in), s, batch_lens);
    prof.end(s);
    for (uint32_t l = 1; l <= last; ++l) {
        void* out = (l == last && final_out != nullptr) ? final_out : buf[l % 2].ptr;
        prof.begin(LK_STAGE_MERGE, static_cast<int>(l), 1,
                   nbatch * (elem(l - 1) * plan.fold_size(l - 1) + elem(l) * plan.fold_size(l)) +
                       coord_bytes(l),
                   s);
        const uint64_t n_inner = plan.param_counts[l][plan.nparams - 1];
        merge_level(in, out, level_coords(l), taylor, n_inner, plan.ncoords[l] / n_inner,
                    plan.ncoords[l - 1], plan.nsegments[l] * nbatch, nbins, s, is_bf16(l - 1),
                    is_bf16(l), merge_pb);
        prof.end(s);
        in = out;
    }
    *last_bf16 = is_bf16(last);
    return in;
}

void FFAExec::execute(const float* ts_e, const float* ts_v, float* fold, uint64_t fold_len,
                      cudaStream_t s, uint64_t nbatch) {
    const uint32_t L = plan.n_levels;
    require(fold_len >= plan.fold_size(L - 1) * nbatch, "fold must hold fold_size floats");
    DeviceGuard g(device);
    prof.reset();
    bool bf16 = false;
    run_levels(ts_e, ts_v, L - 1, fold, s, nbatch, &bf16);
}

void FFAExec::scores(const float* ts_e, const float* ts_v, float* d_scores, uint64_t len,
                     cudaStream_t s, uint64_t nbatch) {
    const uint32_t L = plan.n_levels;
    require(plan.nsegments[L - 1] == 1, "compute_ffa_scores: nsegments must be 1 for scores");
    require(len >= plan.ncoords[L - 1] * plan.widths.size() * nbatch,
            "scores must hold ncoords * n_widths floats");
    DeviceGuard g(device);
    prof.reset();
    scores_impl(ts_e, ts_v, d_scores, nullptr, s, nbatch);
}

void FFAExec::scores_impl(const float* ts_e, const float* ts_v, float* d_scores, float* d_cmax,
                          cudaStream_t s, uint64_t nbatch, float count_thr, uint32_t* d_counts) {
    const uint32_t L = plan.n_levels;
    bool in_bf16 = false;
    const void* in = run_levels(ts_e, ts_v, L - 2, nullptr, s, nbatch, &in_bf16);
    const uint64_t nscores = plan.ncoords[L - 1] * plan.widths.size();
    prof.begin(LK_STAGE_MERGE_SCORE, static_cast<int>(L - 1), 1,
               nbatch * ((in_bf16 ? 2 : 4) * plan.fold_size(L - 2) + 4 * nscores) +
                   coord_bytes(L - 1),
               s);
    const uint64_t n_inner = plan.param_counts[L - 1][plan.nparams - 1];
    if (use_wm()) {
        merge_score_level_wm(in, level_coords(L - 1), plan.nparams > 1, n_inner,
                             plan.ncoords[L - 1] / n_inner, plan.ncoords[L - 2],
                             static_cast<uint32_t>(plan.cfg.nbins), mp, LK_SCORE_PER_WIDTH,
                             d_scores, s, nbatch, in_bf16, d_cmax, normtab.as<float>(), count_thr,
                             d_counts, score_cells == 0);
    } else {
        require(d_counts == nullptr, "internal: block counts need the masked final level");
        merge_score_level(in, level_coords(L - 1), plan.nparams > 1, n_inner,
                          plan.ncoords[L - 1] / n_inner, plan.ncoords[L - 2],
                          static_cast<uint32_t>(plan.cfg.nbins), sp, LK_SCORE_PER_WIDTH, d_scores,
                          s, nbatch, in_bf16, d_cmax, score_cells);
    }
    prof.end(s);
}

void FFAExec::search(const float* ts_e, const float* ts_v, float snr_min, uint32_t* d_idx,
                     float* d_snr, uint64_t max_cands, uint64_t* d_count, cudaStream_t s,
                     uint64_t nbatch) {
    const uint32_t L = plan.n_levels;
    require(plan.nsegments[L - 1] == 1, "compute_ffa_scores: nsegments must be 1 for scores");
    require(nbatch >= 1 && nbatch <= max_batch, "nbatch must lie in [1, max_batch]");
    const uint64_t ncells = plan.ncoords[L - 1] * nbatch;
    const uint64_t n = ncells * plan.widths.size();
    DeviceGuard g(device);
    if (scores_tmp.bytes < n * sizeof(float)) {
        scores_tmp.alloc(n * sizeof(float));
        compact_scratch.alloc(compact_scratch_bytes(n));
    }
    if (mixed && cmax.bytes < ncells * sizeof(float)) {
        cmax.alloc(ncells * sizeof(float));
        cells.alloc(ncells * sizeof(uint32_t));
        cell_vals.alloc(ncells * sizeof(float));
        cell_count.alloc(sizeof(uint64_t));
        cell_scratch.alloc(compact_scratch_bytes(ncells));
    }
    prof.reset();
    if (!mixed && use_wm()) {
        // The final level counts each block's candidates; the list is the
        // scan of the counts and a scatter of the blocks that have any.
        const uint64_t n_inner = plan.param_counts[L - 1][plan.nparams - 1];
        const uint64_t n_outer = plan.ncoords[L - 1] / n_inner;
        const uint64_t nblk = final_level_blocks(n_inner, n_outer, nbatch);
        if (blk_counts.bytes < nblk * sizeof(uint32_t)) {
            blk_counts.alloc(nblk * sizeof(uint32_t));
            blk_offsets.alloc(nblk * sizeof(uint64_t));
        }
        scores_impl(ts_e, ts_v, scores_tmp.as<float>(), nullptr, s, nbatch, snr_min,
                    blk_counts.as<uint32_t>());
        prof.begin(LK_STAGE_COMPACT, -1, 2, 12 * nblk, s);
        compact_ranges(scores_tmp.as<float>(), blk_counts.as<uint32_t>(), blk_offsets.as<uint64_t>(),
                       n_inner, n_outer, nbatch, static_cast<uint32_t>(plan.widths.size()), snr_min,
                       d_idx, d_snr, max_cands, d_count, s);
        prof.end(s);
        return;
    }
    scores_impl(ts_e, ts_v, scores_tmp.as<float>(), mixed ? cmax.as<float>() : nullptr, s, nbatch);
    if (mixed) {
        // Cells whose approximate best S/N is near or above snr_min get their
        // exact FP32 scores; every other cell stays below snr_min.
        prof.begin(LK_STAGE_COMPACT, static_cast<int>(L - 1), 3, 8 * ncells, s);
        compact_ge(cmax.as<float>(), ncells, rescore_threshold(snr_min), cells.as<uint32_t>(),
                   cell_vals.as<float>(), ncells, cell_count.as<uint64_t>(), cell_scratch.ptr, s);
        prof.end(s);
        prof.begin(LK_STAGE_RESCORE, -1, 1, 0, s);
        rescore_cells(fold0.as<float>(), rtree, plan.nparams > 1, sp, cells.as<uint32_t>(),
                      cell_count.as<uint64_t>(), ncells, scores_tmp.as<float>(), s);
        prof.end(s);
    }
    prof.begin(LK_STAGE_COMPACT, -1, 3, 8 * n, s);
    compact_ge(scores_tmp.as<float>(), n, snr_min, d_idx, d_snr, max_cands, d_count,
               compact_scratch.ptr, s);
    prof.end(s);
}

uint64_t FFAExec::rescored_cells(cudaStream_t s) {
    if (!mixed || cell_count.ptr == nullptr) {
        return 0;
    }
    DeviceGuard g(device);
    LK_CUDA(cudaStreamSynchronize(s));
    uint64_t c = 0;
    LK_CUDA(cudaMemcpy(&c, cell_count.ptr, sizeof(c), cudaMemcpyDeviceToHost));
    return c;
}

namespace {

// Sum of the recorded stage times of the given kinds (after a synchronise).
float stage_ms(const StageProfiler& prof, std::initializer_list<int> kinds) {
    float total = 0.0f;
    for (size_t i = 0; i < prof.used; ++i) {
        const auto& st = prof.stages[i];
        for (int k : kinds) {
            if (st.kind == k) {
                float ms = 0.0f;
                LK_CUDA(cudaEventElapsedTime(&ms, st.start, st.stop));
                total += ms;
            }
        }
    }
    return total;
}

}  // namespace

void FFAExec::apply_tuning(const lk_tuning& t) {
    DeviceGuard g(device);
    require(t.merge_rows_in_flight >= 0 && t.merge_rows_in_flight <= 16,
            "merge rows in flight must lie in [0, 16]");
    if (t.bf_rows != 0 || t.bf_warps != 0 || t.bf_stages != 0 || t.bf_tmem_warps != 0) {
        require(bf->configure(t.bf_rows != 0 ? t.bf_rows : bf->rows(), t.bf_warps,
                              t.bf_stages != 0 ? t.bf_stages : bf->stages(), t.bf_tmem_warps),
                "brute-fold launch shape does not fit this plan");
    }
    merge_pb = t.merge_rows_in_flight;
    score_cells = t.score_cells_per_block;
    tuning = t;
    tuning.bf_rows = bf->rows();
    tuning.bf_warps = bf->warps();
    tuning.bf_stages = bf->stages();
    tuning.bf_tmem_warps = bf->tmem_warps();
}

lk_tuning FFAExec::autotune(const float* ts_e, const float* ts_v, uint32_t reps,
                            cudaStream_t s) {
    // A scoring plan (one final segment) is timed through the fused final
    // level; a plan that stops at several segments (the pruning input) through
    // its levels alone, and has no final-level step.
    const bool scoring = plan.nsegments[plan.n_levels - 1] == 1;
    DeviceGuard g(device);
    reps = std::max<uint32_t>(1, std::min<uint32_t>(reps, 20));
    const uint64_t n = plan.ncoords[plan.n_levels - 1] * plan.widths.size();
    if (scoring && scores_tmp.bytes < n * sizeof(float)) {
        scores_tmp.alloc(n * sizeof(float));
        compact_scratch.alloc(compact_scratch_bytes(n));
    }
    const bool was_enabled = prof.enabled;
    prof.enabled = true;
    // the candidates are timed on the caller's single series, in full
    const uint64_t* saved_lens = batch_lens;
    batch_lens = nullptr;
    lk_tuning best{};
    uint32_t tried = 0;
    // Median of reps timed passes (after one untimed pass) of the stages.
    auto time_stages = [&](std::initializer_list<int> kinds) {
        std::vector<float> t;
        for (uint32_t r = 0; r <= reps; ++r) {
            prof.reset();
            if (scoring) {
                scores_impl(ts_e, ts_v, scores_tmp.as<float>(), nullptr, s, 1);
            } else {
                bool last_bf16 = false;
                run_levels(ts_e, ts_v, plan.n_levels - 1, nullptr, s, 1, &last_bf16);
            }
            LK_CUDA(cudaStreamSynchronize(s));
            if (r > 0) {
                t.push_back(stage_ms(prof, kinds));
            }
        }
        std::sort(t.begin(), t.end());
        ++tried;
        return t[t.size() / 2];
    };
    try {
        // 1. brute fold (with the interleave pass when both rows share a warp)
        const uint32_t rows0 = bf->rows(), warps0 = bf->warps(), stages0 = bf->stages();
        float bf_best = INFINITY;
        uint32_t br = rows0, bw = warps0, bs = stages0;
        // best packed (two-row) shared-memory shape, the base of step 1b
        float pk_best = INFINITY;
        uint32_t pw = 0, ps = stages0;
        for (uint32_t rows = 1; rows <= 2; ++rows) {
            if (rows == 2 && plan.cfg.nbins > 128) {
                continue;
            }
            for (uint32_t stages = 2; stages <= 4; ++stages) {
                const uint32_t wmax = bf->max_warps(rows, stages);
                if (wmax == 0) {
                    continue;
                }
                std::vector<uint32_t> ws{0};
                for (uint32_t w = wmax; w >= std::max<uint32_t>(1, (3 * wmax + 3) / 4); --w) {
                    ws.push_back(w);
                    if (w == 1) {
                        break;
                    }
                }
                for (uint32_t w : ws) {
                    if (!bf->configure(rows, w, stages)) {
                        continue;
                    }
                    const float ms = time_stages({LK_STAGE_INTERLEAVE, LK_STAGE_BRUTE_FOLD});
                    if (ms < bf_best) {
                        bf_best = ms;
                        br = rows;
                        bw = bf->warps();
                        bs = stages;
                    }
                    if (rows == 2 && ms < pk_best) {
                        pk_best = ms;
                        pw = bf->warps();
                        ps = stages;
                    }
                }
            }
        }
        // 1b. tensor-memory warps added to the best shared-memory shape
        // (the warps of a block share the sample ring, so a block's time
        // follows its slowest warp; a few shared-memory warp counts below the
        // best are tried with each TMEM warp count, for whole waves of blocks)
        // The base is the best two-row shape even when one row per warp was
        // faster: with nbins above 64 few two-row warps fit shared memory
        // alone, and the TMEM warps are what make the packed form pay.
        uint32_t bt = 0;
        if (pw > 0) {
            const uint32_t ws0 = pw;
            for (uint32_t t = 4; t <= 16; t += 4) {
                for (uint32_t ws = ws0 > 4 ? ws0 - 4 : 1; ws <= ws0; ++ws) {
                    if (t > bf->max_tmem_warps(ws) || !bf->configure(2, ws + t, ps, t)) {
                        continue;
                    }
                    const float ms = time_stages({LK_STAGE_INTERLEAVE, LK_STAGE_BRUTE_FOLD});
                    if (ms < bf_best) {
                        bf_best = ms;
                        bt = t;
                        br = 2;
                        bw = ws;
                        bs = ps;
                    }
                }
            }
        }
        require(bf->configure(br, bw + bt, bs, bt), "autotune: lost the brute-fold shape");
        // 2. merges
        const uint32_t nb = static_cast<uint32_t>(plan.cfg.nbins);
        std::vector<int> pbs{0};
        if (nb == 32) {
            pbs = {4, 8, 16};
        } else if (nb == 64) {
            pbs = {2, 4, 8};
        } else if (nb == 128) {
            pbs = {1, 2, 4};
        }
        float merge_best = INFINITY;
        int bpb = 0;
        // levels 1 .. L-2 are plain merges when scoring, 1 .. L-1 otherwise
        if (plan.n_levels > (scoring ? 2u : 1u)) {
            for (int pb : pbs) {
                merge_pb = pb;
                const float ms = time_stages({LK_STAGE_MERGE});
                if (ms < merge_best) {
                    merge_best = ms;
                    bpb = pb;
                }
            }
        } else {
            merge_best = 0.0f;
        }
        merge_pb = bpb;
        // 3. fused final level: cells per block
        const uint32_t rs = sc::row_stride(nb, sp.wmax);
        const uint32_t tmax = sc::profiles_per_block(rs);
        float score_best = scoring ? INFINITY : 0.0f;
        uint32_t bcells = 0;
        if (scoring && wm) {
            // masked final level (final_level.cu), with and without the table
            for (uint32_t v : {0u, 1u}) {
                score_cells = v;
                const float ms = time_stages({LK_STAGE_MERGE_SCORE});
                if (ms < score_best) {
                    score_best = ms;
                    bcells = v;
                }
            }
        }
        for (uint32_t cells = 32; scoring && cells <= tmax; cells += 32) {
            score_cells = cells;
            const float ms = time_stages({LK_STAGE_MERGE_SCORE});
            if (ms < score_best) {
                score_best = ms;
                bcells = cells;
            }
        }
        score_cells = bcells;
        best.bf_rows = br;
        best.bf_warps = bf->warps();
        best.bf_stages = bs;
        best.bf_tmem_warps = bt;
        best.merge_rows_in_flight = bpb;
        best.score_cells_per_block = bcells;
        best.candidates = tried;
        best.bf_ms = bf_best;
        best.merge_ms = merge_best;
        best.score_ms = score_best;
    } catch (...) {
        prof.enabled = was_enabled;
        prof.reset();
        batch_lens = saved_lens;
        throw;
    }
    prof.enabled = was_enabled;
    prof.reset();
    batch_lens = saved_lens;
    tuning = best;
    return best;
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
