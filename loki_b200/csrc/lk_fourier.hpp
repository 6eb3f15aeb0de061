// Fourier-domain FFA executor (internal): FFACUDA<ComplexTypeCUDA> of the
// reference (lib/ffa_cuda.cu, lib/ffa.cpp:75-135,170-310). Kernels in
// fourier.cu.
#pragma once

#include <memory>
#include <vector>

#include "lk_ffa.hpp"
#include "lk_kernels.hpp"

namespace lk {

// PulsarSearchConfig's nbins_min_lossy_bf default (include/loki/search/
// configs.hpp:37): above it the level-0 fold is the time-domain brute fold
// followed by a real transform instead of the direct transform.
constexpr uint64_t kNbinsMinLossy = 64;

// Level-0 direct transform of segments (kernels::brute_fold_ts_complex,
// lib/kernels.cpp:1156-1242): out [nseg][nfreq][2][nbf] complex.
void fourier_dft_fold(const float* d_ts_e, const float* d_ts_v, const double* d_freqs,
                      uint32_t nfreq, uint64_t seglen, uint64_t nseg, uint32_t nbins, double tsamp,
                      double t_ref, float2* d_out, cudaStream_t s);
// One merge level in the Fourier domain (kernels::ffa_complex_iter[_freq],
// lib/kernels.cpp:942-1130): fractional shifts as phase rotations.
void fourier_merge_level(const float2* d_in, float2* d_out, const void* d_coords, bool taylor,
                         uint64_t ncur, uint64_t nprev, uint64_t nseg, uint32_t nbins,
                         cudaStream_t s);
// Batched real transforms of size nbins over nprof profiles (FFTW's r2c
// unscaled; c2r scaled by 1 / nbins, as math::irfft_batch).
void rfft_profiles(const float* d_in, float2* d_out, uint64_t nprof, uint32_t nbins,
                   cudaStream_t s);
void irfft_profiles(const float2* d_in, float* d_out, uint64_t nprof, uint32_t nbins,
                    cudaStream_t s);

// Final level fused with the inverse transform and the boxcar scorer
// (nbins <= 64, one final segment): scores [ncur][nwidths].
bool fourier_final_supported(uint32_t nbins);
uint32_t fourier_final_jcount(uint32_t nbins);
std::vector<float2> fourier_final_twiddles(uint32_t nbins);
void fourier_final_score(const float2* d_in, const void* d_coords, bool taylor, uint64_t ncur,
                         uint64_t nprev, uint32_t nbins, const ScoreParams& sp, const float2* d_tw,
                         float* d_scores, cudaStream_t s);

// The same level-0 transform on the tensor cores (fourier_mma.cu): three
// FP16 tcgen05.mma passes over hi / lo halves, FP32 accumulation. Needs
// nbins / 2 <= 64 harmonics and segment lengths that are multiples of 8.
bool fourier_mma_supported(uint64_t seglen, uint64_t nseg, uint32_t nbins);
struct FourierMma {
    uint64_t seglen, nseg;
    uint32_t nbins, nfreq;
    uint32_t ntile = 0, nsub = 0, ngroups = 0, tmem_cols = 0;
    uint32_t cpp = 0, nparts = 1;  // K chunks per part, parts (partial folds summed in FP32)
    size_t smem_bytes = 0;
    DeviceBuffer hi, lo, dc, aux;  // FP16 staging [2 nseg][seglen], row sums, max / exponents
    DeviceBuffer parts;            // [nparts][level-0 fold] partial folds (nparts > 1)
    CUtensorMap map_hi{}, map_lo{};
    // max_sub: MMA column subtiles of 256 per block (2: both rows E and V of
    // 256 segments in one block, one block per SM; 1: two blocks per SM);
    // part_chunks: K chunks of 32 samples per part at most (a multiple of 8)
    FourierMma(uint64_t seglen, uint64_t nseg, uint32_t nbins, uint32_t nfreq, uint32_t max_sub = 2,
               uint32_t part_chunks = 64);
    uint64_t device_bytes() const;
    void run(const float* d_ts_e, const float* d_ts_v, const double* d_freqs, double tsamp,
             double t_ref, float2* d_out, uint32_t* d_status, cudaStream_t s);
};

struct FourierExec {
    Plan plan;
    int device;
    uint32_t nbf;        // nbins / 2 + 1
    bool lossy = false;  // level 0 by time-domain brute fold + real transform
    StageProfiler prof;
    DeviceBuffer status;  // brute-fold status word (lossy path)
    DeviceBuffer coords;  // all levels, reference layout
    DeviceBuffer freqs0;  // level-0 frequencies (double)
    DeviceBuffer buf[2];  // complex ping-pong levels
    DeviceBuffer tfold;   // lossy: level-0 time-domain fold
    DeviceBuffer tfinal;  // final fold back in time (scores / search)
    DeviceBuffer scores_tmp, compact_scratch;
    DeviceBuffer final_tw;  // twiddles of the fused final level (nbins <= 64)
    std::unique_ptr<BruteFoldDevice> bf;  // lossy path only
    std::unique_ptr<FourierMma> mma;      // tensor-core level 0 (when the shape allows)
    // Level-0 kernel of the direct transform: LK_FOURIER_L0_AUTO (tensor cores
    // when supported), _CUDA_CORES or _TENSOR_CORES.
    int level0 = LK_FOURIER_L0_AUTO;
    ScoreParams sp{};

    FourierExec(const Plan& p, int device, uint64_t nbins_min_lossy);
    uint64_t fold_size(uint32_t level) const {
        return plan.nsegments[level] * plan.ncoords[level] * 2 * nbf;
    }
    uint64_t fold_size_time(uint32_t level) const { return plan.fold_size(level); }
    uint64_t device_bytes() const;
    const void* level_coords(uint32_t l) const;
    // Levels 0 .. n_levels - 1; the final level lands in final_out when given
    // (else in a ping-pong buffer). Returns the final complex fold.
    // last_level < 0: the final level.
    const float2* run_levels(const float* ts_e, const float* ts_v, float2* final_out,
                             cudaStream_t s, int last_level = -1);
    void execute(const float* ts_e, const float* ts_v, float2* fold, uint64_t len_complex,
                 cudaStream_t s);
    void execute_time(const float* ts_e, const float* ts_v, float* fold, uint64_t len,
                      cudaStream_t s);
    void scores(const float* ts_e, const float* ts_v, float* d_scores, uint64_t len,
                cudaStream_t s);
    void search(const float* ts_e, const float* ts_v, float snr_min, uint32_t* d_idx, float* d_snr,
                uint64_t max_cands, uint64_t* d_count, cudaStream_t s);
    std::vector<lk_stage_time> profile(cudaStream_t s);
    void set_level0(int mode);
    // Times the tensor-core level 0's tilings (subtiles per block, K part
    // length) on these series and keeps the fastest; results agree to FP32
    // accuracy whichever is kept. Returns the kept level-0 time (ms).
    float tune_level0(const float* ts_e, const float* ts_v, uint32_t reps, cudaStream_t s);
    bool uses_mma() const { return mma != nullptr && level0 != LK_FOURIER_L0_CUDA_CORES; }
    uint32_t read_status(cudaStream_t s);

private:
    void scores_into(const float* ts_e, const float* ts_v, float* d_scores, cudaStream_t s);
};

}  // namespace lk
