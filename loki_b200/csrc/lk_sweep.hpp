// FFAFreqSweep: region planner and executor (sweep.cpp).
#pragma once

#include <memory>
#include <vector>

#include "lk_ffa.hpp"
#include "lk_fourier.hpp"
#include "lk_internal.hpp"
#include "lk_kernels.hpp"

namespace lk {

struct FFAExec;

// coord::FFARegion (include/loki/common/coord.hpp): one octave of the sweep.
struct SweepRegion {
    double f_start, f_end;
    uint64_t nbins;
    double eta;
};

// The planner's knobs (PulsarSearchConfig defaults of the reference).
struct SweepOptions {
    double max_memory_gb = 8.0;           // max_process_memory_gb
    double octave_scale = 2.0;
    uint64_t nbins_max = 1024;
    uint64_t max_passing_candidates = 1ull << 22;
    bool decode_chunk_widths = false;  // false: the reference's decode (base widths)
    bool device_memory_model = true;   // FFAFreqSweepCUDA's model; false: FFAFreqSweep's
    int executor_mode = 0;             // 0 auto, 1 resident, 2 one chunk at a time
    bool autotune = false;             // tune each chunk executor's launch shapes once
    bool use_fourier = false;          // chunks through the Fourier-domain FFA
    uint64_t nbins_min_lossy_bf = 64;  // Fourier chunks: lossy level 0 above this nbins
    int plan_sizes = 0;  // 0 as the executors need, 1 FFARegionPlanner<float>, 2 <ComplexType>
};

// One chunk: its configuration (drift-widened frequency limits, the region's
// nbins and eta), nominal range and the plan sizes behind the memory model.
struct SweepChunk {
    lk_config cfg;
    double nominal_f_start, nominal_f_end;
    uint64_t buffer_size, coord_size, ncoords, n_levels;
    double memory_gb;     // this chunk alone
    double allocated_gb;  // with the largest sizes of the chunks before it
};

std::vector<SweepRegion> generate_ffa_regions(double p_min, double p_max, double tsamp,
                                              uint64_t nbins_min, double eta_min,
                                              double octave_scale, uint64_t nbins_max);
std::vector<SweepChunk> plan_freq_sweep(const lk_config& base, const SweepOptions& opt);

// One chunk's executor: the time-domain FFA, or the Fourier-domain FFA.
struct ChunkExec {
    std::unique_ptr<FFAExec> t;
    std::unique_ptr<FourierExec> f;
    const Plan& plan() const { return t ? t->plan : f->plan; }
    StageProfiler& prof() { return t ? t->prof : f->prof; }
    std::vector<lk_stage_time> profile(cudaStream_t s) { return t ? t->profile(s) : f->profile(s); }
    void search(const float* ts_e, const float* ts_v, float snr_min, uint32_t* d_idx, float* d_snr,
                uint64_t max_cands, uint64_t* d_count, cudaStream_t s) {
        if (t) {
            t->search(ts_e, ts_v, snr_min, d_idx, d_snr, max_cands, d_count, s);
        } else {
            f->search(ts_e, ts_v, snr_min, d_idx, d_snr, max_cands, d_count, s);
        }
    }
};

class FreqSweepExec {
public:
    FreqSweepExec(const lk_config& base, const SweepOptions& opt, int device, int storage);
    ~FreqSweepExec();
    // Every chunk: FFA + scores + compaction `>= snr_min` + parameter decode.
    // Chunks run on two internal streams after the work already queued on
    // `s`; synchronises `s` twice (counts, then candidates).
    void execute(const float* d_ts_e, const float* d_ts_v, cudaStream_t s);
    const std::vector<SweepChunk>& chunks() const { return m_chunks; }
    const std::vector<double>& params() const { return m_params; }   // [n][nparams + 1]
    const std::vector<float>& scores() const { return m_scores; }
    const std::vector<uint64_t>& region_counts() const { return m_region_counts; }
    uint32_t nparams() const { return m_base.nparams; }
    // Stage timing of every chunk's executor (CUDA events); profile() sums
    // the last execute's stages by kind over levels and chunks (level -1).
    void set_profiling(bool enable);
    std::vector<lk_stage_time> profile(cudaStream_t s);

private:
    ChunkExec& exec(size_t i);
    // exec(i), its launch shapes tuned on (or restored for) these series
    // (time-domain chunks)
    ChunkExec& tuned_exec(size_t i, const float* d_ts_e, const float* d_ts_v, cudaStream_t s);
    lk_config m_base;
    SweepOptions m_opt;
    int m_device, m_storage;
    std::vector<SweepChunk> m_chunks;
    std::vector<uint32_t> m_base_widths;
    std::vector<std::unique_ptr<ChunkExec>> m_execs;
    DeviceBuffer m_idx, m_snr, m_cnt;
    std::vector<double> m_params;
    std::vector<float> m_scores;
    std::vector<uint64_t> m_region_counts;
    bool m_profiling = false;
    int m_mode = 0;  // 0 undecided, 1 every chunk's executor resident, 2 one chunk at a time
    std::vector<lk_tuning> m_tunings;  // per chunk, once tuned
    std::vector<bool> m_tuned;
    std::vector<lk_stage_time> m_prof;  // summed by kind during execute
    static constexpr int kSweepStreams = 2;  // chunks alternate between them
    std::vector<cudaStream_t> m_streams;
    std::vector<cudaEvent_t> m_done;
    cudaEvent_t m_ready = nullptr;
};

}  // namespace lk
