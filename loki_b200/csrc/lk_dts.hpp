// DynamicThresholdScheme on the GPU (internal): host set-up restated from the
// reference and the executor of the beam search (kernels in dts.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "lk_ffa.hpp"
#include "lk_internal.hpp"
#include "lk_kernels.hpp"
#include "loki_b200.h"

namespace lk {

// Entries of the normal quantile table (ThreadLocalNormalRNG's 2^17 + 1).
constexpr uint32_t kDtsLutSize = (1u << 17) + 1;

// Inverse standard normal CDF in double: Acklam's rational approximation
// (P. J. Acklam, 2003) refined by one Halley step on erfc.
double normal_quantile(double p);
// Normal quantile table: quantile(clamp(i / 2^17, 1e-9, 1 - 1e-9)) as float.
std::vector<float> normal_lut();

// Host set-up of DynamicThresholdScheme (lib/thresholds.cpp:560-606,
// lib/scheme.cpp, lib/simulation.cpp, lib/utils.cpp:138-185).
std::vector<float> dts_thresholds(float snr_start, float snr_final, uint32_t n);
std::vector<float> dts_probs(uint32_t nprobs, float prob_min);
std::vector<float> dts_profile(uint32_t nbins, float ducy, float center);
std::vector<float> dts_guess_scheme(uint32_t nstages, float snr_bound,
                                    const std::vector<float>& branching, uint32_t trials_start,
                                    float min_trials);
std::vector<uint32_t> dts_neighbours(const std::vector<uint32_t>& indices, uint32_t target,
                                     uint32_t num);
int64_t dts_lower_bin(const std::vector<float>& range, float value);
lk_dts_state dts_state_initial();
lk_dts_state dts_state_empty();
lk_dts_state dts_gen_next(const lk_dts_state& s, float threshold, float success_h0,
                          float success_h1, float nbranches);

// One transition of a stage: threshold index, the previous stage's cell it
// starts from, and its identifier in the noise counter space.
struct DtsTrans {
    uint32_t ithres;
    uint32_t prev_cell;
    uint32_t tid;
    uint32_t pad;
};

class DtsExec {
public:
    DtsExec(const lk_dts_config& cfg, int device);
    // Runs the whole scheme on `s` (stage 0 from the initial folds, then
    // every later stage) and copies the states back (synchronises `s`).
    void run(uint32_t thres_neigh, cudaStream_t s);

    uint32_t nstages() const { return static_cast<uint32_t>(m_branching.size()); }
    uint32_t nthresholds() const { return static_cast<uint32_t>(m_thresholds.size()); }
    uint32_t nprobs() const { return static_cast<uint32_t>(m_probs.size()); }
    uint32_t nbins() const { return m_nbins; }
    std::vector<uint32_t> beam(uint32_t istage) const;
    std::vector<float> best_path(float min_pd) const;
    uint64_t device_bytes() const;

    std::vector<float> m_branching, m_profile, m_thresholds, m_probs, m_guess;
    std::vector<uint32_t> m_widths;
    std::vector<lk_dts_state> m_states;  // [nstages][nthresholds][nprobs], after run
    float m_bias_snr = 0.0f;
    uint64_t m_transitions = 0;  // transitions the last run simulated

private:
    uint32_t m_nbins, m_ntrials;
    float m_beam_width;
    uint64_t m_seed;
    int m_device;
    ScoreParams m_sp{};
    DeviceBuffer m_lut, m_prof2, m_thr_dev, m_probs_dev, m_init_pool, m_init_state, m_init_counts;
    DeviceBuffer m_pool[2], m_counts[2], m_states_dev, m_trans, m_beam_dev, m_toff, m_nsurv,
        m_winner, m_status, m_work;
};

}  // namespace lk
