// FFAFreqSweep: the reference's production caller of the FFA path.
//
// Region planner (lib/regions.cpp:31-78, 166-514): the frequency range is cut
// into octave regions whose nbins grows with the period (constant bin width
// in time, constant duty-cycle resolution eta / nbins), and each region into
// chunks small enough for the memory budget: the largest chunk ending at the
// current upper edge is found by bisection over its width, with each
// chunk's frequency range widened by the largest Doppler drift the other
// parameters allow. Executor (lib/ffa_freq_sweep.cpp:76-269): per chunk, FFA
// + boxcar scores + ordered `>= snr_min` compaction, then every passing
// (coordinate, width) decoded into parameter values by the chunk plan's
// Cartesian strides.
//
// The memory models are the reference's (FFARegionStats, float arithmetic
// as there: the process model of FFAFreqSweep or the device model of
// FFAFreqSweepCUDA), so the chunk boundaries -- and with them the candidate
// list -- are the reference's.
#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>
#include <vector>

#include "lk_ffa.hpp"
#include "lk_sweep.hpp"

namespace lk {

namespace {

constexpr uint64_t kWriteBatchSize = 1u << 16;  // kFFAFreqSweepWriteBatchSize

// FFARegionStats::get_cpu_memory_usage (lib/regions.cpp:101-135), in GB.
float cpu_memory_gb(uint64_t buf, uint64_t coord, uint64_t nc, uint64_t n_widths,
                    uint32_t n_params, uint64_t max_passing, uint64_t fold_bytes) {
    const float gib = static_cast<float>(1ull << 30);
    const float buffer = static_cast<float>(2 * buf * fold_bytes) / gib;
    const uint64_t coord_bytes = coord * (n_params == 1 ? 8 : 16);
    const float coords = static_cast<float>(coord_bytes) / gib;
    const uint64_t scores = std::max(nc * n_widths, max_passing);
    const uint64_t write_sets = kWriteBatchSize * (n_params + 1);
    const float extra = static_cast<float>((write_sets * sizeof(double)) +
                                           (scores * sizeof(uint32_t)) + (scores * sizeof(float))) /
                        gib;
    return buffer + coords + extra;
}

// FFARegionStats::get_device_memory_usage (lib/regions.cpp:136-149), in GB:
// the input series, scores and passing indices on the device, then the fold
// buffers and coordinates.
float device_memory_gb(uint64_t buf, uint64_t coord, uint64_t nc, uint64_t n_widths,
                       uint32_t n_params, uint64_t nsamps, uint64_t max_passing, uint64_t fold_bytes) {
    const float gib = static_cast<float>(1ull << 30);
    const uint64_t scores = std::max(nc * n_widths, max_passing);
    const float extra = static_cast<float>((((2 * nsamps) + scores) * sizeof(float)) +
                                           (scores * sizeof(uint32_t))) /
                        gib;
    const float buffer = static_cast<float>(2 * buf * fold_bytes) / gib;
    const uint64_t coord_bytes = coord * (n_params == 1 ? 8 : 16);
    const float coords = static_cast<float>(coord_bytes) / gib;
    return extra + buffer + coords;
}

// calculate_max_drift (lib/regions.cpp:179-204).
double max_drift(const lk_config& c) {
    if (c.nparams <= 1) {
        return 0.0;
    }
    const double t_half = (static_cast<double>(c.nsamps) * c.tsamp) / 2.0;
    auto amax = [&](uint32_t i) {
        return std::max(std::abs(c.param_limits[2 * i]), std::abs(c.param_limits[2 * i + 1]));
    };
    if (c.nparams == 2) {
        return (amax(0) * t_half) / kCval;
    }
    if (c.nparams == 3) {
        const double max_jerk = amax(0), max_accel = amax(1);
        return ((max_accel * t_half) + (max_jerk * t_half * t_half / 2.0)) / kCval;
    }
    fail(LK_ERR_UNSUPPORTED, "Unsupported number of parameters for drift calculation");
}

}  // namespace

std::vector<SweepRegion> generate_ffa_regions(double p_min, double p_max, double tsamp,
                                              uint64_t nbins_min, double eta_min,
                                              double octave_scale, uint64_t nbins_max) {
    require(p_min > 0.0, "p_min must be positive.");
    require(p_max > p_min, "p_max must be > p_min.");
    require(tsamp > 0.0, "tsamp must be positive.");
    require(nbins_min >= 2, "nbins_min must be >= 2.");
    require(eta_min > 0.0, "eta_min must be positive.");
    require(octave_scale >= 1.0, "octave_scale must be >= 1.0.");
    require(nbins_max >= nbins_min, "nbins_max must be >= nbins_min.");
    std::vector<SweepRegion> regions;
    uint64_t nbins_cur = std::min(nbins_min, static_cast<uint64_t>(p_min / tsamp));
    const double rho = eta_min / static_cast<double>(nbins_cur);
    const double bin_width = p_min / static_cast<double>(nbins_cur);
    double p_cur_low = p_min;
    while (p_cur_low < p_max) {
        const uint64_t nbins_k = nbins_cur;
        if (nbins_k >= nbins_max) {
            const double eta_k = std::round(rho * static_cast<double>(nbins_max));
            regions.push_back({1.0 / p_max, 1.0 / p_cur_low, nbins_max, eta_k});
            break;
        }
        const double p_cur_high = std::min(p_cur_low * octave_scale, p_max);
        const double eta_k = rho * static_cast<double>(nbins_k);
        regions.push_back({1.0 / p_cur_high, 1.0 / p_cur_low, nbins_k, eta_k});
        p_cur_low = p_cur_high;
        nbins_cur = static_cast<uint64_t>(p_cur_low / bin_width);
    }
    return regions;
}

std::vector<SweepChunk> plan_freq_sweep(const lk_config& base, const SweepOptions& opt) {
    require(base.nparams >= 1 && base.nparams <= 3, "the frequency sweep supports nparams 1 to 3");
    const uint32_t np = base.nparams;
    const double f_min = base.param_limits[2 * (np - 1)];
    const double f_max = base.param_limits[2 * (np - 1) + 1];
    require(f_min > 0.0 && f_max > f_min, "frequency limits must satisfy 0 < f_min < f_max");
    const Plan base_plan = make_plan(base, /*sizes_only=*/true);
    const uint64_t n_widths = base_plan.widths.size();
    const auto regions = generate_ffa_regions(1.0 / f_max, 1.0 / f_min, base.tsamp, base.nbins,
                                              base.eta, opt.octave_scale, opt.nbins_max);
    const double drift = max_drift(base);
    if (drift < 0.0 || drift >= 1.0) {
        fail(LK_ERR_INVALID_ARG,
             "FFARegionPlanner: max_drift must be in [0, 1); the parameter range is too large "
             "for the observation duration");
    }
    const double effective_limit_gb = opt.max_memory_gb - 0.5;  // kSafetyMarginGB
    require(effective_limit_gb > 0.0,
            "FFARegionPlanner: max_process_memory_gb must exceed the 0.5 GB safety margin");
    constexpr double kRelativeTolerance = 1.0e-4;
    constexpr double kAbsoluteToleranceHz = 1.0e-2;
    constexpr uint64_t kMaxBisectionSteps = 50;
    constexpr double kSliverWidthFactor = 4.0;

    // get_freq_sweep_memory_usage: the device model for FFAFreqSweepCUDA, the
    // process model for FFAFreqSweep.
    // fold elements are complex harmonics (8 bytes) for the Fourier-domain FFA
    const uint64_t fold_bytes = opt.use_fourier ? 8 : sizeof(float);
    auto memory_gb = [&](uint64_t buf, uint64_t coord, uint64_t nc) -> double {
        if (opt.device_memory_model) {
            return device_memory_gb(buf, coord, nc, n_widths, np, base.nsamps,
                                    opt.max_passing_candidates, fold_bytes);
        }
        return cpu_memory_gb(buf, coord, nc, n_widths, np, opt.max_passing_candidates, fold_bytes);
    };
    std::vector<SweepChunk> chunks;
    uint64_t mbuf = 0, mcoord = 0, mnc = 0, mlv = 0;
    for (const auto& rg : regions) {
        const double f_start = rg.f_start, f_end = rg.f_end;
        if (f_end <= f_start) {
            continue;
        }
        if (f_start * (1.0 - drift) <= 0.0) {
            fail(LK_ERR_INVALID_ARG,
                 "FFARegionPlanner: drift expansion would push f_start to a non-positive "
                 "frequency");
        }
        const double region_span = f_end - f_start;
        const double tol = std::max(kAbsoluteToleranceHz, kRelativeTolerance * region_span);
        // evaluate_chunk: the drift-widened configuration and its sizes
        auto evaluate = [&](double nominal_start, double nominal_end) {
            require(nominal_end > nominal_start, "FFARegionPlanner: zero/negative-width chunk");
            const double actual_start = nominal_start * (1.0 - drift);
            const double actual_end = nominal_end * (1.0 + drift);
            require(actual_start > 0.0 && actual_end > actual_start,
                    "FFARegionPlanner: invalid drift-expanded range");
            SweepChunk ch{};
            ch.cfg = base;
            ch.cfg.nbins = rg.nbins;
            ch.cfg.eta = rg.eta;
            ch.cfg.param_limits[2 * (np - 1)] = actual_start;
            ch.cfg.param_limits[2 * (np - 1) + 1] = actual_end;
            const Plan pl = make_plan(ch.cfg, /*sizes_only=*/true);
            ch.nominal_f_start = nominal_start;
            ch.nominal_f_end = nominal_end;
            // FFAPlan<ComplexType>::get_buffer_size counts nbins / 2 + 1 harmonics per row
            const bool complex_sizes =
                opt.plan_sizes == 2 || (opt.plan_sizes == 0 && opt.use_fourier);
            ch.buffer_size = complex_sizes ? pl.buffer_size / rg.nbins * (rg.nbins / 2 + 1)
                                           : pl.buffer_size;
            ch.coord_size = pl.coord_size;
            ch.ncoords = pl.ncoords.back();
            ch.n_levels = pl.n_levels;
            ch.memory_gb = memory_gb(ch.buffer_size, ch.coord_size, ch.ncoords);
            ch.allocated_gb = memory_gb(std::max(mbuf, ch.buffer_size),
                                        std::max(mcoord, ch.coord_size),
                                        std::max(mnc, ch.ncoords));
            return ch;
        };
        auto fits = [&](const SweepChunk& c) { return c.allocated_gb <= effective_limit_gb; };
        double cur_end = f_end;
        while (cur_end > f_start) {
            // find_largest_fitting_chunk
            const double remaining = cur_end - f_start;
            double nominal_start;
            SweepChunk ev = evaluate(f_start, cur_end);
            if (fits(ev)) {
                nominal_start = f_start;
            } else {
                const double min_width = std::min(remaining, kAbsoluteToleranceHz);
                SweepChunk min_ev = evaluate(cur_end - min_width, cur_end);
                if (!fits(min_ev)) {
                    fail(LK_ERR_INVALID_ARG,
                         "FFARegionPlanner: Cannot fit minimum viable chunk; increase "
                         "max_memory_gb or reduce parameter search ranges");
                }
                double lo_w = min_width, hi_w = remaining;
                SweepChunk best = min_ev;
                for (uint64_t step = 0; step < kMaxBisectionSteps && (hi_w - lo_w) > tol; ++step) {
                    const double mid_w = (lo_w + hi_w) / 2.0;
                    SweepChunk probe = evaluate(cur_end - mid_w, cur_end);
                    if (fits(probe)) {
                        lo_w = mid_w;
                        best = probe;
                    } else {
                        hi_w = mid_w;
                    }
                }
                nominal_start = cur_end - lo_w;
                ev = best;
                // try_absorb_sliver
                const double rem = nominal_start - f_start;
                if (rem > 0.0 && rem <= kSliverWidthFactor * tol) {
                    SweepChunk merged = evaluate(f_start, cur_end);
                    if (fits(merged)) {
                        nominal_start = f_start;
                        ev = merged;
                    }
                }
            }
            if (nominal_start >= cur_end) {
                fail(LK_ERR_INTERNAL, "FFARegionPlanner: no progress (planner bug)");
            }
            ev.nominal_f_start = nominal_start;
            ev.nominal_f_end = cur_end;
            chunks.push_back(ev);
            mbuf = std::max(mbuf, ev.buffer_size);
            mcoord = std::max(mcoord, ev.coord_size);
            mnc = std::max(mnc, ev.ncoords);
            mlv = std::max(mlv, ev.n_levels);
            cur_end = nominal_start;
        }
    }
    return chunks;
}

FreqSweepExec::FreqSweepExec(const lk_config& base, const SweepOptions& opt, int device,
                             int storage)
    : m_base(base), m_opt(opt), m_device(device), m_storage(storage) {
    m_chunks = plan_freq_sweep(base, opt);
    m_base_widths = make_plan(base, /*sizes_only=*/true).widths;
    m_execs.resize(m_chunks.size());
}

ChunkExec& FreqSweepExec::exec(size_t i) {
    if (!m_execs[i]) {
        auto c = std::make_unique<ChunkExec>();
        if (m_opt.use_fourier) {
            c->f = std::make_unique<FourierExec>(make_plan(m_chunks[i].cfg), m_device,
                                                 m_opt.nbins_min_lossy_bf);
        } else {
            c->t = std::make_unique<FFAExec>(make_plan(m_chunks[i].cfg), m_device, m_storage);
        }
        c->prof().enabled = m_profiling;
        m_execs[i] = std::move(c);
    }
    return *m_execs[i];
}

ChunkExec& FreqSweepExec::tuned_exec(size_t i, const float* d_ts_e, const float* d_ts_v,
                                     cudaStream_t s) {
    const bool fresh = !m_execs[i];
    ChunkExec& cx = exec(i);
    if (!m_opt.autotune || !cx.t) {
        return cx;
    }
    FFAExec& ex = *cx.t;
    if (m_tuned.size() != m_chunks.size()) {
        m_tuned.assign(m_chunks.size(), false);
        m_tunings.assign(m_chunks.size(), lk_tuning{});
    }
    if (!m_tuned[i]) {
        m_tunings[i] = ex.autotune(d_ts_e, d_ts_v, 3, s);
        m_tuned[i] = true;
    } else if (fresh) {
        ex.apply_tuning(m_tunings[i]);
    }
    return cx;
}

void FreqSweepExec::set_profiling(bool enable) {
    m_profiling = enable;
    for (auto& e : m_execs) {
        if (e) {
            e->prof().enabled = enable;
            e->prof().reset();
        }
    }
    m_prof.clear();
}

std::vector<lk_stage_time> FreqSweepExec::profile(cudaStream_t /*s*/) { return m_prof; }

void FreqSweepExec::execute(const float* d_ts_e, const float* d_ts_v, cudaStream_t s) {
    DeviceGuard g(m_device);
    const uint32_t np = m_base.nparams;
    const size_t nch = m_chunks.size();
    // Every chunk gets room for all of its cells (the reference's scores
    // buffer holds max(max_ncoords * n_widths, max_passing_candidates)), so a
    // chunk never overflows; chunks are searched concurrently, each into its
    // own region.
    std::vector<uint64_t> off(nch + 1, 0), cap(nch, 0);
    for (size_t i = 0; i < nch; ++i) {
        const auto& c = m_chunks[i];
        const uint64_t nw = m_base.n_score_widths > 0
                                ? m_base.n_score_widths
                                : box_width_trials(c.cfg.nbins, c.cfg.ducy_max, c.cfg.wtsp).size();
        cap[i] = std::max<uint64_t>(1, c.ncoords * nw);
        off[i + 1] = off[i] + cap[i];
    }
    // Every chunk's executor stays resident (its tables reused by the next
    // sweep, chunks overlapping on two streams) when all of them fit in free
    // device memory with room to spare; otherwise the chunks run one at a
    // time, each executor released after its chunk, so the device never holds
    // more than one chunk's workspace (the planner's memory budget).
    if (m_mode == 0 && (m_opt.executor_mode == 1 || m_opt.executor_mode == 2)) {
        m_mode = m_opt.executor_mode;
    }
    if (m_mode == 0) {
        double total_gb = 0.0;
        for (const auto& c : m_chunks) {
            total_gb += c.memory_gb;
        }
        size_t free_b = 0, total_b = 0;
        LK_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const double free_gb = static_cast<double>(free_b) / static_cast<double>(1ull << 30);
        m_mode = (1.25 * total_gb <= 0.8 * free_gb) ? 1 : 2;
    } else if (m_mode == 1 && m_opt.executor_mode == 0) {
        // Chosen automatically on an earlier execute: executors that are not
        // resident yet (an earlier execute stopped part-way) are checked
        // against the free memory of now; once all are resident, nothing more
        // is allocated and the mode stays.
        double missing_gb = 0.0;
        for (size_t i = 0; i < nch; ++i) {
            if (i >= m_execs.size() || !m_execs[i]) {
                missing_gb += m_chunks[i].memory_gb;
            }
        }
        if (missing_gb > 0.0) {
            size_t free_b = 0, total_b = 0;
            LK_CUDA(cudaMemGetInfo(&free_b, &total_b));
            const double free_gb = static_cast<double>(free_b) / static_cast<double>(1ull << 30);
            if (1.25 * missing_gb > 0.8 * free_gb) {
                m_mode = 2;
            }
        }
    }
    const bool resident = m_mode == 1;
    uint64_t need = 0;
    for (size_t i = 0; i < nch; ++i) {
        need = resident ? off[i + 1] : std::max(need, cap[i]);
    }
    if (m_idx.bytes < std::max<uint64_t>(1, need) * sizeof(uint32_t)) {
        m_idx.alloc(std::max<uint64_t>(1, need) * sizeof(uint32_t));
        m_snr.alloc(std::max<uint64_t>(1, need) * sizeof(float));
    }
    if (m_cnt.bytes < std::max<size_t>(1, nch) * sizeof(uint64_t)) {
        m_cnt.alloc(std::max<size_t>(1, nch) * sizeof(uint64_t));
    }
    if (m_streams.empty()) {
        m_streams.resize(kSweepStreams);
        m_done.resize(kSweepStreams);
        for (int k = 0; k < kSweepStreams; ++k) {
            LK_CUDA(cudaStreamCreateWithFlags(&m_streams[k], cudaStreamNonBlocking));
            LK_CUDA(cudaEventCreateWithFlags(&m_done[k], cudaEventDisableTiming));
        }
        LK_CUDA(cudaEventCreateWithFlags(&m_ready, cudaEventDisableTiming));
    }
    m_params.clear();
    m_scores.clear();
    m_region_counts.assign(nch, 0);
    m_prof.clear();
    // `score >= snr_min` compares the float score promoted to double: the
    // same set as `score >= thr` with thr the smallest float not below snr_min.
    float thr = static_cast<float>(m_base.snr_min);
    if (static_cast<double>(thr) < m_base.snr_min) {
        thr = std::nextafter(thr, std::numeric_limits<float>::infinity());
    }
    std::vector<uint64_t> counts(nch, 0);
    std::vector<std::vector<uint32_t>> h_idx(nch);
    std::vector<std::vector<float>> h_snr(nch);
    std::vector<Plan> plans(nch);
    auto add_profile = [&](ChunkExec& ex, cudaStream_t st_of) {
        for (const lk_stage_time& st : ex.profile(st_of)) {
            auto it = std::find_if(m_prof.begin(), m_prof.end(),
                                   [&](const lk_stage_time& a) { return a.kind == st.kind; });
            if (it == m_prof.end()) {
                lk_stage_time a = st;
                a.level = -1;
                m_prof.push_back(a);
            } else {
                it->launches += st.launches;
                it->ms += st.ms;
                it->bytes += st.bytes;
            }
        }
    };
    // Counts and candidates of chunks [i0, i1), region off[i] - base.
    auto read_back = [&](size_t i0, size_t i1, uint64_t base) {
        LK_CUDA(cudaMemcpyAsync(counts.data() + i0, m_cnt.as<uint64_t>() + i0,
                                (i1 - i0) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        LK_CUDA(cudaStreamSynchronize(s));
        for (size_t i = i0; i < i1; ++i) {
            require(counts[i] <= cap[i], "FFAFreqSweep: candidate buffer overflow");
            h_idx[i].resize(counts[i]);
            h_snr[i].resize(counts[i]);
            if (counts[i] > 0) {
                LK_CUDA(cudaMemcpyAsync(h_idx[i].data(), m_idx.as<uint32_t>() + (off[i] - base),
                                        counts[i] * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
                LK_CUDA(cudaMemcpyAsync(h_snr[i].data(), m_snr.as<float>() + (off[i] - base),
                                        counts[i] * sizeof(float), cudaMemcpyDeviceToHost, s));
            }
        }
        LK_CUDA(cudaStreamSynchronize(s));
    };
    auto check_plan = [](const ChunkExec& ex) {
        require(ex.plan().nsegments[ex.plan().n_levels - 1] == 1,
                "FFAFreqSweep::execute_ffa_region: nsegments must be 1 to call scoring function");
    };
    if (resident) {
        // Chunks alternate between two streams: one chunk's brute fold runs
        // beside the previous chunk's merges and scoring. The executors are
        // built first (allocations synchronise the device).
        for (size_t i = 0; i < nch; ++i) {
            check_plan(tuned_exec(i, d_ts_e, d_ts_v, s));
        }
        LK_CUDA(cudaEventRecord(m_ready, s));
        for (int k = 0; k < kSweepStreams; ++k) {
            LK_CUDA(cudaStreamWaitEvent(m_streams[k], m_ready, 0));
        }
        for (size_t i = 0; i < nch; ++i) {
            m_execs[i]->search(d_ts_e, d_ts_v, thr, m_idx.as<uint32_t>() + off[i],
                               m_snr.as<float>() + off[i], cap[i], m_cnt.as<uint64_t>() + i,
                               m_streams[i % kSweepStreams]);
        }
        for (int k = 0; k < kSweepStreams; ++k) {
            LK_CUDA(cudaEventRecord(m_done[k], m_streams[k]));
            LK_CUDA(cudaStreamWaitEvent(s, m_done[k], 0));
        }
        if (nch > 0) {
            read_back(0, nch, 0);
        }
        for (size_t i = 0; i < nch; ++i) {
            if (m_profiling) {
                add_profile(*m_execs[i], m_streams[i % kSweepStreams]);
            }
            plans[i] = m_execs[i]->plan();
        }
    } else {
        for (size_t i = 0; i < nch; ++i) {
            ChunkExec& ex = tuned_exec(i, d_ts_e, d_ts_v, s);
            check_plan(ex);
            ex.search(d_ts_e, d_ts_v, thr, m_idx.as<uint32_t>(), m_snr.as<float>(), cap[i],
                      m_cnt.as<uint64_t>() + i, s);
            read_back(i, i + 1, off[i]);
            if (m_profiling) {
                add_profile(ex, s);
            }
            plans[i] = ex.plan();
            m_execs[i].reset();  // release this chunk's workspace
        }
    }
    for (size_t i = 0; i < nch; ++i) {
        const Plan& pl = plans[i];
        const uint32_t L = pl.n_levels - 1;
        const uint64_t total = counts[i];
        m_region_counts[i] = total;
        // save_results (lib/ffa_freq_sweep.cpp:202-250): decode with the
        // chunk plan's final-level counts and Cartesian strides and (by
        // default) the base configuration's width list, as the reference
        // does.
        const std::vector<uint32_t>& dec_widths =
            m_opt.decode_chunk_widths ? pl.widths : m_base_widths;
        const uint64_t nw_dec = dec_widths.size();
        std::vector<uint64_t> pc(np), strides(np);
        for (uint32_t j = 0; j < np; ++j) {
            pc[j] = pl.param_counts[L][j];
        }
        strides[np - 1] = 1;
        for (int j = static_cast<int>(np) - 2; j >= 0; --j) {
            strides[j] = strides[j + 1] * pc[j + 1];
        }
        for (uint64_t k = 0; k < total; ++k) {
            const uint64_t score_idx = h_idx[i][k];
            const uint64_t coord_idx = score_idx / nw_dec;
            const uint64_t width_idx = score_idx % nw_dec;
            uint64_t rem = coord_idx;
            for (uint32_t j = 0; j < np; ++j) {
                const uint64_t pidx = rem / strides[j];
                rem -= pidx * strides[j];
                const double vmin = pl.lim_min(j), vmax = pl.lim_max(j);
                double val;
                if (pc[j] <= 1) {
                    val = (vmax + vmin) / 2.0;
                } else {
                    const double dv = (vmax - vmin) / static_cast<double>(pc[j]);
                    val = vmin + (dv * (static_cast<double>(pidx) + 0.5));
                }
                m_params.push_back(val);
            }
            m_params.push_back(static_cast<double>(dec_widths[width_idx]));
            m_scores.push_back(h_snr[i][k]);
        }
    }
}

FreqSweepExec::~FreqSweepExec() {
    if (!m_streams.empty()) {
        DeviceGuard g(m_device);
        for (int k = 0; k < kSweepStreams; ++k) {
            cudaStreamSynchronize(m_streams[k]);
            cudaEventDestroy(m_done[k]);
            cudaStreamDestroy(m_streams[k]);
        }
        cudaEventDestroy(m_ready);
    }
}

}  // namespace lk
