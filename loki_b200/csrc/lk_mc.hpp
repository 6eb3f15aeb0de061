// Host side of the Monte-Carlo threshold stage (kernels in mc.cu).
#pragma once

#include <cstdint>

#include "lk_ffa.hpp"
#include "lk_internal.hpp"
#include "lk_kernels.hpp"

#define LK_MC_MAX_THRESHOLDS 64

namespace lk {

// One stage's inputs and outputs (device pointers unless noted).
struct McStage {
    const float* d_folds_in = nullptr;   // [ntrials_in][nbins]
    uint64_t ntrials_in = 0;
    const uint32_t* d_src = nullptr;     // NULL: trial i reads input row i
    uint64_t ntrials = 0;
    uint64_t nrows = 0;                  // rows of d_noise (and of a per-trial d_signal)
    const float* d_noise = nullptr;      // rows indexed by rowmap[i] (or i)
    const float* d_signal = nullptr;     // [nbins], or per trial when signal_per_trial
    bool signal_per_trial = false;
    float signal_scale = 1.0f;
    const uint32_t* d_rowmap = nullptr;  // NULL: identity
    float var_in = 0.0f;
    float var_add = 1.0f;
    float threshold = 0.0f;
    const float* thresholds = nullptr;   // host, n_thr entries
    uint32_t n_thr = 0;
    float* d_folds_out = nullptr;        // [ntrials][nbins] (survivors first)
    uint32_t* d_ids_out = nullptr;       // optional: noise row of each survivor
    uint64_t* d_count = nullptr;         // survivors
    const uint8_t* d_class = nullptr;    // optional: class flag per noise row
    uint64_t* d_counts = nullptr;        // [n_thr] (+ [n_thr] for flagged rows when d_class)
    float* d_max_snr = nullptr;          // optional: [ntrials] max S/N per trial
};

class McExec {
public:
    McExec(uint64_t max_trials, uint32_t nbins, const uint32_t* widths, uint32_t nwidths,
           int device);
    void stage(const McStage& st, cudaStream_t s);
    // Synchronises `s`, returns and clears the bad-index flag word.
    uint32_t read_status(cudaStream_t s);
    uint64_t device_bytes() const;

private:
    uint64_t m_max;
    uint32_t m_nbins;
    int m_device;
    ScoreParams m_sp{};
    DeviceBuffer m_max_snr, m_idx, m_vals, m_scratch, m_thr, m_status;
    DeviceBuffer m_stage_folds;  // [max_trials][nbins]: every trial's fold of the stage
};

}  // namespace lk
