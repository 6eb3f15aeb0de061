// DynamicThresholdScheme beam search on the GPU.
//
// Reference: DynamicThresholdScheme::Impl (lib/thresholds.cpp:560-907):
// init_states simulates the initial H0 / H1 folds and the stage-0
// transitions; run_segment, for every later stage, takes each threshold of
// the stage's beam, each of its neighbouring thresholds in the previous
// beam and each probability bin, and runs simulate_score_prune_fused on the
// H0 and H1 folds of that previous state (lib/thresholds.cpp:358-431):
//   out_i   = (in[src_i] + noise_i) + profile * bias      (src_i = i, or a
//             uniformly drawn survivor once i passes the survivors)
//   survive = some width's boxcar S/N / sqrt(var_in + 1) > threshold
// then State::gen_next (include/loki/detection/thresholds.hpp:32-58) and, in
// the state's probability bin, keeps the first transition with the smallest
// complexity_cumul.
//
// B200 layout: every transition of a stage is independent, so one launch
// simulates and scores all of them at once and only counts survivors (no
// fold is written); one thread per beam threshold then replays that
// threshold's transitions in the reference's order and keeps the winner of
// each cell, which is the reference's update rule with no lock (a cell is
// only ever written by transitions of its own threshold); a last launch
// rebuilds the winners' folds -- the noise is a function of (stage,
// transition, trial, bin), so the rebuilt folds are the counted ones -- and
// stores the survivors in trial order for the next stage. The whole scheme
// runs without a host synchronisation until the states are read back.
//
// Noise: the reference's generator (ThreadLocalNormalRNG,
// lib/loki/math.hpp:229-420) maps 32-bit uniforms through a 2^17 + 1 entry
// table of normal quantiles with linear interpolation (fmaf), and resamples
// with Lemire's bounded method; both are kept. Its uniforms come from
// thread-local PCG32 streams seeded from std::random_device, which no
// parallel schedule can reproduce; here each uniform is a Philox4x32-10 word
// (Salmon et al., SC 2011) of the counter (trial, bin / 4, transition * 2 +
// hypothesis, stage + 1) under a 64-bit seed, so every run, every launch
// shape and the CPU oracle draw the same numbers.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>
#include <numbers>
#include <stdexcept>

#include "lk_block.cuh"
#include "lk_device.cuh"
#include "lk_dts.hpp"
#include "lk_score.cuh"

namespace lk {

// ---- host set-up ----------------------------------------------------------

double normal_quantile(double p) {
    // Acklam's coefficients (lower / central / upper regions).
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02,
                                -2.759285104469687e+02, 1.383577518672690e+02,
                                -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02,
                                -1.556989798598866e+02, 6.680131188771972e+01,
                                -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01,
                                -2.400758277161838e+00, -2.549732539343734e+00,
                                4.374664141464968e+00,  2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01,
                                2.445134137142996e+00, 3.754408661907416e+00};
    const double p_low = 0.02425;
    double x;
    if (p < p_low) {
        const double q = std::sqrt(-2.0 * std::log(p));
        x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    } else if (p <= 1.0 - p_low) {
        const double q = p - 0.5;
        const double r = q * q;
        x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
            (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
    } else {
        const double q = std::sqrt(-2.0 * std::log(1.0 - p));
        x = -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    }
    // One Halley step: e = Phi(x) - p.
    const double e = 0.5 * std::erfc(-x / std::sqrt(2.0)) - p;
    const double u = e * std::sqrt(2.0 * 3.14159265358979323846) * std::exp(x * x / 2.0);
    return x - u / (1.0 + x * u / 2.0);
}

std::vector<float> normal_lut() {
    // ThreadLocalNormalRNG::init_lut (lib/loki/math.hpp:304-312).
    std::vector<float> lut(kDtsLutSize);
    const double n = static_cast<double>(kDtsLutSize - 1);
    for (uint32_t i = 0; i < kDtsLutSize; ++i) {
        double p = static_cast<double>(i) / n;
        p = std::clamp(p, 1e-9, 1.0 - 1e-9);
        lut[i] = static_cast<float>(normal_quantile(p));
    }
    return lut;
}

// detail::compute_thresholds (lib/scheme.cpp:16-25).
std::vector<float> dts_thresholds(float snr_start, float snr_final, uint32_t n) {
    std::vector<float> t(n);
    const float step = (snr_final - snr_start) / static_cast<float>(n - 1);
    for (uint32_t i = 0; i < n; ++i) {
        t[i] = (static_cast<float>(i) * step) + snr_start;
    }
    return t;
}

// detail::compute_probs (lib/scheme.cpp:27-40).
std::vector<float> dts_probs(uint32_t nprobs, float prob_min) {
    require(nprobs > 1, "Number of probabilities must be > 1");
    require(prob_min < 1.0f && prob_min > 0.0f, "Probability must lie in (0, 1)");
    std::vector<float> p(nprobs);
    const float log_prob_min = std::log10(prob_min);
    const float step = (0.0F - log_prob_min) / static_cast<float>(nprobs - 1);
    for (uint32_t i = 0; i < nprobs; ++i) {
        p[i] = std::pow(10.0F, log_prob_min + (step * static_cast<float>(i)));
    }
    return p;
}

// simulation::generate_folded_profile (lib/simulation.cpp:12-50).
std::vector<float> dts_profile(uint32_t nbins, float ducy, float center) {
    std::vector<float> out(nbins);
    const float step = 1.0F / static_cast<float>(nbins);
    const float sigma = ducy / (2.0F * std::sqrt(2.0F * std::numbers::ln10_v<float>));
    for (uint32_t i = 0; i < nbins; ++i) {
        const float p = static_cast<float>(i) * step;
        const float wrapped = std::fmod(p - center + 0.5F, 1.0F) - 0.5F;
        out[i] = std::exp(-(wrapped * wrapped) / (2.0F * sigma * sigma));
    }
    const float max_val = *std::max_element(out.begin(), out.end());
    for (float& v : out) {
        v = v / max_val;
    }
    float ss = 0.0F;
    for (float v : out) {
        ss = ss + v * v;
    }
    const float norm = std::sqrt(ss);
    for (float& v : out) {
        v = v / norm;
    }
    return out;
}

// detail::bound_scheme / trials_scheme / guess_scheme (lib/scheme.cpp:56-96);
// norm_isf(p) = -quantile(p).
std::vector<float> dts_guess_scheme(uint32_t nstages, float snr_bound,
                                    const std::vector<float>& branching, uint32_t trials_start,
                                    float min_trials) {
    std::vector<float> out(nstages);
    const uint32_t nsegments = nstages + 1;
    float log2_trials = std::log2(static_cast<float>(trials_start));
    for (uint32_t i = 0; i < nstages; ++i) {
        const float bound = std::sqrt(static_cast<float>(i + 2) * snr_bound * snr_bound /
                                      static_cast<float>(nsegments));
        log2_trials += std::log2(branching[i]);
        const float trials = std::exp2(log2_trials);
        const float eff = std::max(trials, min_trials);
        const float thr = static_cast<float>(-normal_quantile(static_cast<double>(1 / eff)));
        out[i] = std::min(bound, thr);
    }
    return out;
}

// utils::find_neighbouring_indices (lib/utils.cpp:138-163).
std::vector<uint32_t> dts_neighbours(const std::vector<uint32_t>& indices, uint32_t target,
                                     uint32_t num) {
    require(!indices.empty(), "find_neighbouring_indices: indices empty");
    require(num > 0, "find_neighbouring_indices: num == 0");
    const auto it = std::lower_bound(indices.begin(), indices.end(), target);
    const auto pos = static_cast<uint64_t>(it - indices.begin());
    const uint64_t half = num / 2;
    uint64_t left = pos > half ? pos - half : 0;
    const uint64_t right = std::min<uint64_t>(indices.size(), left + num);
    if (right - left < num && right == indices.size()) {
        left = right > num ? right - num : 0;
    }
    return std::vector<uint32_t>(indices.begin() + static_cast<int64_t>(left),
                                 indices.begin() + static_cast<int64_t>(right));
}

// utils::find_lower_bin_index (lib/utils.cpp:181-185).
int64_t dts_lower_bin(const std::vector<float>& range, float value) {
    const auto it = std::upper_bound(range.begin(), range.end(), value);
    return static_cast<int64_t>(it - range.begin()) - 1;
}

lk_dts_state dts_state_empty() {
    lk_dts_state s{};
    s.success_h0 = 0.0f;
    s.success_h1 = 0.0f;
    s.complexity = 0.0f;
    s.complexity_cumul = std::numeric_limits<float>::max();
    s.success_h1_cumul = 0.0f;
    s.nbranches = 0.0f;
    s.threshold = -1.0f;
    s.cost = std::numeric_limits<float>::max();
    s.threshold_prev = -1.0f;
    s.success_h1_cumul_prev = 0.0f;
    s.is_empty = 1;
    return s;
}

lk_dts_state dts_state_initial() {
    lk_dts_state s = dts_state_empty();
    s.complexity = 1.0f;
    s.complexity_cumul = 1.0f;
    s.success_h1_cumul = 1.0f;
    s.is_empty = 0;
    return s;
}

// State::gen_next (include/loki/detection/thresholds.hpp:32-58); host and
// device share the formula.
__host__ __device__ __forceinline__ lk_dts_state gen_next_hd(const lk_dts_state& s, float threshold,
                                                             float success_h0, float success_h1,
                                                             float nbranches) {
#ifdef __CUDA_ARCH__
    const float nleaves_next = __fmul_rn(s.complexity, nbranches);
    const float nleaves_surv = __fmul_rn(nleaves_next, success_h0);
    const float cc_next = __fadd_rn(s.complexity_cumul, nleaves_next);
    const float h1_next = __fmul_rn(s.success_h1_cumul, success_h1);
    const float cost_next = __fdiv_rn(cc_next, h1_next);
#else
    const float nleaves_next = s.complexity * nbranches;
    const float nleaves_surv = nleaves_next * success_h0;
    const float cc_next = s.complexity_cumul + nleaves_next;
    const float h1_next = s.success_h1_cumul * success_h1;
    const float cost_next = cc_next / h1_next;
#endif
    lk_dts_state n{};
    n.success_h0 = success_h0;
    n.success_h1 = success_h1;
    n.complexity = nleaves_surv;
    n.complexity_cumul = cc_next;
    n.success_h1_cumul = h1_next;
    n.nbranches = nbranches;
    n.threshold = threshold;
    n.cost = cost_next;
    n.is_empty = 0;
    n.threshold_prev = s.threshold;
    n.success_h1_cumul_prev = s.success_h1_cumul;
    return n;
}

lk_dts_state dts_gen_next(const lk_dts_state& s, float threshold, float success_h0,
                          float success_h1, float nbranches) {
    return gen_next_hd(s, threshold, success_h0, success_h1, nbranches);
}

// ---- device --------------------------------------------------------------

namespace {

constexpr uint32_t kWarp = 32;
constexpr uint32_t kStatusTally = 1u << 11;  // rebuilt survivors differ from the counted ones

struct Philox {
    uint32_t v[4];
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC 2011).
__host__ __device__ __forceinline__ Philox philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2,
                                                         uint32_t c3, uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return {{c0, c1, c2, c3}};
}

// generate_impl of ThreadLocalNormalRNG (lib/loki/math.hpp:363-390) for one
// uniform word: table index and fraction, fmaf interpolation, then
// fmaf(z, stddev, mean) with stddev 1 and mean 0.
__device__ __forceinline__ float normal_of(uint32_t r, const float* __restrict__ lut) {
    constexpr float kInvU32 = 1.0F / 4294967296.0F;  // 1.0F / float(UINT32_MAX)
    constexpr float kMaxIdx = static_cast<float>(kDtsLutSize - 2);
    const float u = __fmul_rn(__fmul_rn(__uint2float_rn(r), kInvU32), kMaxIdx);
    const uint32_t idx = __float2uint_rz(u);
    const float frac = __fsub_rn(u, __uint2float_rn(idx));
    const float lo = __ldg(lut + idx);
    const float hi = __ldg(lut + idx + 1);
    const float z = __fmaf_rn(frac, __fsub_rn(hi, lo), lo);
    return __fmaf_rn(z, 1.0f, 0.0f);
}

// uniform_index(range - 1) (lib/loki/math.hpp:267-285): Lemire's bounded
// draw with rejection, on the words of counter (i, ~0 - k, tid2, stage).
__device__ __forceinline__ uint32_t resample_index(uint32_t range, uint32_t i, uint32_t tid2,
                                                   uint32_t stage_code, uint32_t k0, uint32_t k1) {
    const uint64_t t = (1ull << 32) % range;
    uint64_t m = 0;
    for (uint32_t call = 0; call < 2; ++call) {
        const Philox w = philox4x32_10(i, 0xFFFFFFFFu - call, tid2, stage_code, k0, k1);
        for (int q = 0; q < 4; ++q) {
            m = static_cast<uint64_t>(w.v[q]) * range;
            if (static_cast<uint32_t>(m) >= range || static_cast<uint32_t>(m) >= t) {
                return static_cast<uint32_t>(m >> 32);
            }
        }
    }
    return static_cast<uint32_t>(m >> 32);
}

struct DtsArgs {
    const float* lut;
    const float* prof2;       // [2][nbins] profile * bias of H0 (bias 0) and H1
    const float* thresholds;  // [nthresholds]
    const float* probs;       // [nprobs]
    uint32_t nbins, ntrials, nthr, nprobs;
    uint32_t k0, k1;          // Philox key (seed)
    float stdnoise;           // sqrt(var_in + 1) of the stage
    float nbranches;
    uint32_t stage_code;      // stage + 1 (0: initial folds)
    const float* prev_pool;   // [prev cells][2][ntrials][nbins]
    const uint32_t* prev_counts;      // [prev cells][2]
    const lk_dts_state* prev_states;  // [prev cells]
    float* next_pool;
    uint32_t* next_counts;
    lk_dts_state* states;     // this stage's [nthr * nprobs]
    const DtsTrans* trans;
    const uint32_t* beam;     // this stage's beam thresholds
    const uint32_t* toff;     // transitions of beam[b]: [toff[b], toff[b + 1])
    uint32_t nbeam;
    uint32_t* nsurv;          // [ntrans][2]
    int32_t* winner;          // [nthr * nprobs]
    uint32_t* status;
    unsigned long long* work; // transitions simulated (both hypotheses)
};

// Fold of trial i of (transition, hypothesis) into row r (items over bins
// in groups of four, one Philox call per group).
__device__ __forceinline__ void build_quad(const DtsArgs& a, const float* in, uint32_t n_in,
                                           uint32_t h, uint32_t tid2, uint32_t i, uint32_t q,
                                           float* row) {
    const uint32_t src =
        i < n_in ? i : resample_index(n_in, i, tid2, a.stage_code, a.k0, a.k1);
    const Philox w = philox4x32_10(i, q, tid2, a.stage_code, a.k0, a.k1);
    const float* ir = in + static_cast<uint64_t>(src) * a.nbins;
    const float* pr = a.prof2 + h * a.nbins;
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k) {
        const uint32_t j = 4 * q + k;
        if (j < a.nbins) {
            row[j] = __fadd_rn(__fadd_rn(__ldg(ir + j), normal_of(w.v[k], a.lut)), __ldg(pr + j));
        }
    }
}

// Initial folds (simulate_folds from zero folds of variance 0): no scoring.
__global__ void dts_init_kernel(DtsArgs a, float* __restrict__ pool) {
    const uint32_t nq = (a.nbins + 3) / 4;
    const uint64_t n = 2ull * a.ntrials * nq;
    for (uint64_t it = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; it < n;
         it += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t q = static_cast<uint32_t>(it % nq);
        const uint32_t i = static_cast<uint32_t>((it / nq) % a.ntrials);
        const uint32_t h = static_cast<uint32_t>(it / (static_cast<uint64_t>(nq) * a.ntrials));
        const Philox w = philox4x32_10(i, q, h, 0u, a.k0, a.k1);
        float* row = pool + (static_cast<uint64_t>(h) * a.ntrials + i) * a.nbins;
        const float* pr = a.prof2 + h * a.nbins;
#pragma unroll
        for (uint32_t k = 0; k < 4; ++k) {
            const uint32_t j = 4 * q + k;
            if (j < a.nbins) {
                row[j] = __fadd_rn(__fadd_rn(0.0f, normal_of(w.v[k], a.lut)), __ldg(pr + j));
            }
        }
    }
}

__device__ __forceinline__ bool prev_usable(const DtsArgs& a, uint32_t cell) {
    return a.prev_states[cell].is_empty == 0 && a.prev_counts[2 * cell] != 0 &&
           a.prev_counts[2 * cell + 1] != 0;
}

// Pass 1: survivors of every (transition, hypothesis), T trials per block.
// WM > 0: nbins NB with the width mask mp, scored by sc::max_snr_div_wm
// (rows of at least NB + WM + 2 floats, rs even); else sc::max_snr_div_any.
template <int NW, int NB, int WM>
__device__ __forceinline__ float dts_max_snr(float* r, const DtsArgs& a, const ScoreParams& sp,
                                             const MaskScoreParams& mp) {
    if constexpr (WM > 0) {
        return sc::max_snr_div_wm<NB, WM>(r, mp, a.stdnoise);
    } else {
        return sc::max_snr_div_any<NB, NW>(r, a.nbins, a.stdnoise, sp);
    }
}

template <int NW, int NB, int WM>
__global__ void dts_count_kernel(DtsArgs a, uint32_t rs, ScoreParams sp, MaskScoreParams mp) {
    extern __shared__ float rows[];
    __shared__ uint32_t s_cnt;
    const DtsTrans tr = a.trans[blockIdx.y];
    const uint32_t h = blockIdx.z;
    if (!prev_usable(a, tr.prev_cell)) {
        return;  // uniform per block
    }
    if (blockIdx.x == 0 && h == 0 && threadIdx.x == 0) {
        atomicAdd(a.work, 1ull);
    }
    const uint32_t T = blockDim.x;
    const uint32_t i0 = blockIdx.x * T;
    const uint32_t nhere = min(T, a.ntrials - i0);
    const uint32_t n_in = a.prev_counts[2 * tr.prev_cell + h];
    const float* in = a.prev_pool + (static_cast<uint64_t>(tr.prev_cell) * 2 + h) * a.ntrials * a.nbins;
    const uint32_t tid2 = tr.tid * 2 + h;
    const uint32_t nq = (a.nbins + 3) / 4;
    if (threadIdx.x == 0) {
        s_cnt = 0;
    }
    for (uint32_t it = threadIdx.x; it < nhere * nq; it += T) {
        const uint32_t p = it / nq, q = it - (it / nq) * nq;
        build_quad(a, in, n_in, h, tid2, i0 + p, q, rows + static_cast<size_t>(p) * rs);
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const float m = dts_max_snr<NW, NB, WM>(rows + static_cast<size_t>(threadIdx.x) * rs, a, sp, mp);
        if (m > a.thresholds[tr.ithres]) {
            atomicAdd(&s_cnt, 1u);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_cnt != 0) {
        atomicAdd(&a.nsurv[2 * blockIdx.y + h], s_cnt);
    }
}

// State update: thread b replays the transitions of beam threshold b in the
// reference's order (neighbours ascending, then probability bins) and keeps
// each cell's first transition with the smallest complexity_cumul.
__global__ void dts_select_kernel(DtsArgs a) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= a.nbeam) {
        return;
    }
    const uint32_t ithres = a.beam[b];
    const float thr = a.thresholds[ithres];
    const float nt = __uint2float_rn(a.ntrials);
    for (uint32_t t = a.toff[b]; t < a.toff[b + 1]; ++t) {
        const DtsTrans tr = a.trans[t];
        if (!prev_usable(a, tr.prev_cell)) {
            continue;
        }
        const float s0 = __fdiv_rn(__uint2float_rn(a.nsurv[2 * t]), nt);
        const float s1 = __fdiv_rn(__uint2float_rn(a.nsurv[2 * t + 1]), nt);
        const lk_dts_state cur = gen_next_hd(a.prev_states[tr.prev_cell], thr, s0, s1, a.nbranches);
        // find_lower_bin_index: index of the last prob <= value, -1 if none
        int64_t iprob = -1;
        for (uint32_t k = 0; k < a.nprobs; ++k) {
            if (!(cur.success_h1_cumul < a.probs[k])) {
                iprob = k;
            } else {
                break;
            }
        }
        if (iprob < 0) {
            continue;
        }
        const uint32_t cell = ithres * a.nprobs + static_cast<uint32_t>(iprob);
        lk_dts_state& ex = a.states[cell];
        if (ex.is_empty != 0 || cur.complexity_cumul < ex.complexity_cumul) {
            ex = cur;
            a.winner[cell] = static_cast<int32_t>(t);
        }
    }
}

// Pass 2: the winners' folds rebuilt, scored again and their survivors
// stored in trial order; one block per (cell, hypothesis).
template <int NW, int NB, int WM>
__global__ void dts_regen_kernel(DtsArgs a, uint32_t rs, ScoreParams sp, MaskScoreParams mp) {
    extern __shared__ float rows[];
    __shared__ uint32_t ws[32];
    const uint32_t cell = blockIdx.x;
    const uint32_t h = blockIdx.y;
    const int32_t t = a.winner[cell];
    if (t < 0) {
        if (threadIdx.x == 0) {
            a.next_counts[2 * cell + h] = 0;
        }
        return;
    }
    const DtsTrans tr = a.trans[t];
    const uint32_t n_in = a.prev_counts[2 * tr.prev_cell + h];
    const float* in = a.prev_pool + (static_cast<uint64_t>(tr.prev_cell) * 2 + h) * a.ntrials * a.nbins;
    float* out = a.next_pool + (static_cast<uint64_t>(cell) * 2 + h) * a.ntrials * a.nbins;
    const uint32_t tid2 = tr.tid * 2 + h;
    const uint32_t nq = (a.nbins + 3) / 4;
    const float thr = a.thresholds[tr.ithres];
    const uint32_t T = blockDim.x;
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    uint32_t pos = 0;
    for (uint32_t i0 = 0; i0 < a.ntrials; i0 += T) {
        const uint32_t nhere = min(T, a.ntrials - i0);
        for (uint32_t it = threadIdx.x; it < nhere * nq; it += T) {
            const uint32_t p = it / nq, q = it - (it / nq) * nq;
            build_quad(a, in, n_in, h, tid2, i0 + p, q, rows + static_cast<size_t>(p) * rs);
        }
        __syncthreads();
        // the scorer writes prefix sums in place: score a copy of the fold
        // in the row's upper half (rs = twice the scorer's row stride)
        bool keep = false;
        if (threadIdx.x < nhere) {
            float* r = rows + static_cast<size_t>(threadIdx.x) * rs;
            float* cp = r + rs / 2;
            for (uint32_t j = 0; j < a.nbins; ++j) {
                cp[j] = r[j];
            }
            keep = dts_max_snr<NW, NB, WM>(cp, a, sp, mp) > thr;
        }
        uint32_t total;
        const uint32_t before = blk::block_exclusive_scan(keep ? 1u : 0u, ws, &total);
        // rank of every kept trial, then warps copy the kept rows out
        __shared__ uint32_t rank[1024];
        if (threadIdx.x < nhere) {
            rank[threadIdx.x] = keep ? before : 0xFFFFFFFFu;
        }
        __syncthreads();
        for (uint32_t p = warp; p < nhere; p += T / kWarp) {
            const uint32_t rk = rank[p];
            if (rk != 0xFFFFFFFFu) {
                const float* r = rows + static_cast<size_t>(p) * rs;
                float* o = out + static_cast<uint64_t>(pos + rk) * a.nbins;
                for (uint32_t j = lane; j < a.nbins; j += kWarp) {
                    o[j] = r[j];
                }
            }
        }
        pos += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        a.next_counts[2 * cell + h] = pos;
        if (pos != a.nsurv[2 * t + h]) {
            atomicOr(a.status, kStatusTally);
        }
    }
}

}  // namespace

// ---- executor ---------------------------------------------------------------

DtsExec::DtsExec(const lk_dts_config& c, int device)
    : m_nbins(c.nbins), m_ntrials(c.ntrials), m_beam_width(c.beam_width), m_seed(c.seed),
      m_device(device) {
    require(c.nstages >= 1 && c.branching_pattern != nullptr, "Branching pattern is empty");
    require(c.nbins >= 4 && c.nbins <= 1024, "nbins must lie in [4, 1024]");
    require(c.ntrials >= 1 && c.ntrials <= (1u << 20), "ntrials must lie in [1, 2^20]");
    require(c.nthresholds >= 2 && c.nthresholds <= 4096, "nthresholds must lie in [2, 4096]");
    require(c.nprobs >= 2 && c.nprobs <= 256, "nprobs must lie in [2, 256]");
    require(c.trials_start >= 1, "trials_start must be >= 1");
    m_branching.assign(c.branching_pattern, c.branching_pattern + c.nstages);
    m_profile = dts_profile(c.nbins, c.ref_ducy, 0.5F);
    m_thresholds = dts_thresholds(0.1F, c.snr_final, c.nthresholds);
    m_probs = dts_probs(c.nprobs, c.prob_min);
    m_widths = box_width_trials(c.nbins, c.ducy_max, c.wtsp);
    m_bias_snr = c.snr_final / static_cast<float>(std::sqrt(static_cast<double>(c.nstages + 1)));
    m_guess = dts_guess_scheme(c.nstages, c.snr_final, m_branching, c.trials_start, 1E10F);
    m_sp = make_score_params(m_widths.data(), static_cast<uint32_t>(m_widths.size()), c.nbins);

    DeviceGuard g(device);
    const std::vector<float> lut = normal_lut();
    m_lut.alloc(lut.size() * sizeof(float));
    LK_CUDA(cudaMemcpy(m_lut.ptr, lut.data(), lut.size() * sizeof(float), cudaMemcpyHostToDevice));
    std::vector<float> prof2(2 * c.nbins);
    for (uint32_t j = 0; j < c.nbins; ++j) {
        prof2[j] = m_profile[j] * 0.0F;            // H0: bias_snr 0
        prof2[c.nbins + j] = m_profile[j] * m_bias_snr;
    }
    m_prof2.alloc(prof2.size() * sizeof(float));
    LK_CUDA(cudaMemcpy(m_prof2.ptr, prof2.data(), prof2.size() * sizeof(float), cudaMemcpyHostToDevice));
    m_thr_dev.alloc(m_thresholds.size() * sizeof(float));
    LK_CUDA(cudaMemcpy(m_thr_dev.ptr, m_thresholds.data(), m_thresholds.size() * sizeof(float),
                       cudaMemcpyHostToDevice));
    m_probs_dev.alloc(m_probs.size() * sizeof(float));
    LK_CUDA(cudaMemcpy(m_probs_dev.ptr, m_probs.data(), m_probs.size() * sizeof(float),
                       cudaMemcpyHostToDevice));
    const uint64_t ncell = static_cast<uint64_t>(nthresholds()) * nprobs();
    const uint64_t pool_floats = ncell * 2 * static_cast<uint64_t>(c.ntrials) * c.nbins;
    for (int k = 0; k < 2; ++k) {
        m_pool[k].alloc(pool_floats * sizeof(float));
        m_counts[k].alloc(ncell * 2 * sizeof(uint32_t));
    }
    m_init_pool.alloc(2ull * c.ntrials * c.nbins * sizeof(float));
    m_init_counts.alloc(2 * sizeof(uint32_t));
    const uint32_t init_counts[2] = {c.ntrials, c.ntrials};
    LK_CUDA(cudaMemcpy(m_init_counts.ptr, init_counts, sizeof(init_counts), cudaMemcpyHostToDevice));
    const lk_dts_state init = dts_state_initial();
    m_init_state.alloc(sizeof(lk_dts_state));
    LK_CUDA(cudaMemcpy(m_init_state.ptr, &init, sizeof(init), cudaMemcpyHostToDevice));
    m_states_dev.alloc(static_cast<uint64_t>(nstages()) * ncell * sizeof(lk_dts_state));
    m_winner.alloc(ncell * sizeof(int32_t));
    m_status.alloc(sizeof(uint32_t));
    LK_CUDA(cudaMemset(m_status.ptr, 0, sizeof(uint32_t)));
    m_work.alloc(sizeof(unsigned long long));
}

uint64_t DtsExec::device_bytes() const {
    return m_lut.bytes + m_prof2.bytes + m_thr_dev.bytes + m_probs_dev.bytes + m_init_pool.bytes +
           m_init_state.bytes + m_init_counts.bytes + m_pool[0].bytes + m_pool[1].bytes +
           m_counts[0].bytes + m_counts[1].bytes + m_states_dev.bytes + m_trans.bytes +
           m_beam_dev.bytes + m_toff.bytes + m_nsurv.bytes + m_winner.bytes + m_status.bytes +
           m_work.bytes;
}

// get_current_thresholds_idx (lib/thresholds.cpp:807-824).
std::vector<uint32_t> DtsExec::beam(uint32_t istage) const {
    const float guess = m_guess[istage];
    const float lower = std::max(0.0F, guess - m_beam_width);
    const float upper = std::min(m_thresholds.back(), guess + m_beam_width);
    std::vector<uint32_t> r;
    for (uint32_t i = 0; i < m_thresholds.size(); ++i) {
        if (m_thresholds[i] >= lower && m_thresholds[i] <= upper) {
            r.push_back(i);
        }
    }
    return r;
}

void DtsExec::run(uint32_t thres_neigh, cudaStream_t s) {
    require(thres_neigh >= 1, "thres_neigh must be >= 1");
    DeviceGuard g(m_device);
    const uint32_t S = nstages(), NT = nthresholds(), NP = nprobs();
    const uint64_t ncell = static_cast<uint64_t>(NT) * NP;
    // Transitions of every stage in the reference's order, grouped by beam
    // threshold.
    std::vector<DtsTrans> trans;
    std::vector<uint32_t> beams, toffs;
    std::vector<uint64_t> st_trans(S + 1), st_beam(S + 1), st_toff(S + 1);
    std::vector<uint32_t> prev_beam;
    for (uint32_t st = 0; st < S; ++st) {
        st_trans[st] = trans.size();
        st_beam[st] = beams.size();
        st_toff[st] = toffs.size();
        const std::vector<uint32_t> cur = beam(st);
        uint32_t local = 0;
        for (uint32_t ithres : cur) {
            beams.push_back(ithres);
            toffs.push_back(local);
            if (st == 0) {
                trans.push_back({ithres, 0u, ithres, 0u});
                ++local;
                continue;
            }
            for (uint32_t j : dts_neighbours(prev_beam, ithres, thres_neigh)) {
                for (uint32_t k = 0; k < NP; ++k) {
                    trans.push_back({ithres, j * NP + k, (ithres * NT + j) * NP + k, 0u});
                    ++local;
                }
            }
        }
        toffs.push_back(local);
        prev_beam = cur;
    }
    st_trans[S] = trans.size();
    st_beam[S] = beams.size();
    st_toff[S] = toffs.size();
    uint64_t max_trans = 1;
    for (uint32_t st = 0; st < S; ++st) {
        max_trans = std::max<uint64_t>(max_trans, st_trans[st + 1] - st_trans[st]);
    }
    require(max_trans <= 65535, "too many transitions in one stage for the launch grid");
    m_trans.alloc(std::max<size_t>(1, trans.size()) * sizeof(DtsTrans));
    m_beam_dev.alloc(std::max<size_t>(1, beams.size()) * sizeof(uint32_t));
    m_toff.alloc(std::max<size_t>(1, toffs.size()) * sizeof(uint32_t));
    m_nsurv.alloc(static_cast<uint64_t>(std::max<size_t>(1, trans.size())) * 2 * sizeof(uint32_t));
    if (!trans.empty()) {
        LK_CUDA(cudaMemcpyAsync(m_trans.ptr, trans.data(), trans.size() * sizeof(DtsTrans),
                                cudaMemcpyHostToDevice, s));
        LK_CUDA(cudaMemcpyAsync(m_beam_dev.ptr, beams.data(), beams.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, s));
        LK_CUDA(cudaMemcpyAsync(m_toff.ptr, toffs.data(), toffs.size() * sizeof(uint32_t),
                                cudaMemcpyHostToDevice, s));
    }
    LK_CUDA(cudaMemsetAsync(m_nsurv.ptr, 0, m_nsurv.bytes, s));
    // every state starts empty (State{})
    std::vector<lk_dts_state> empty(static_cast<size_t>(S) * ncell, dts_state_empty());
    LK_CUDA(cudaMemcpyAsync(m_states_dev.ptr, empty.data(), empty.size() * sizeof(lk_dts_state),
                            cudaMemcpyHostToDevice, s));
    LK_CUDA(cudaMemsetAsync(m_status.ptr, 0, sizeof(uint32_t), s));
    LK_CUDA(cudaMemsetAsync(m_work.ptr, 0, sizeof(unsigned long long), s));

    DtsArgs a{};
    a.lut = m_lut.as<float>();
    a.prof2 = m_prof2.as<float>();
    a.thresholds = m_thr_dev.as<float>();
    a.probs = m_probs_dev.as<float>();
    a.nbins = m_nbins;
    a.ntrials = m_ntrials;
    a.nthr = NT;
    a.nprobs = NP;
    a.k0 = static_cast<uint32_t>(m_seed);
    a.k1 = static_cast<uint32_t>(m_seed >> 32);
    a.status = m_status.as<uint32_t>();
    a.work = m_work.as<unsigned long long>();
    {
        const uint64_t items = 2ull * m_ntrials * ((m_nbins + 3) / 4);
        const auto blocks = static_cast<unsigned>(std::min<uint64_t>((items + 255) / 256, 148ull * 16));
        a.stage_code = 0;
        dts_init_kernel<<<blocks, 256, 0, s>>>(a, m_init_pool.as<float>());
        LK_CUDA(cudaGetLastError());
    }
    // the masked scorer (nbins 32 / 64 / 128, strictly increasing widths <=
    // 32) takes even rows of NB + WM + 2 floats; the generic one odd rows
    MaskScoreParams mp{};
    const bool masked = make_mask_score_params(m_sp, m_nbins, &mp);
    const uint32_t wm = mp.wmax <= 8 ? 8u : (mp.wmax <= 16 ? 16u : 32u);
    const uint32_t rs = masked ? m_nbins + wm + 2 : sc::row_stride(m_nbins, m_sp.wmax);
    const uint32_t T = 128;
    const size_t smem_count = static_cast<size_t>(T) * rs * sizeof(float);
    const uint32_t TR = 128;  // trials per tile in the rebuild (rows hold a fold and its copy)
    const uint32_t rs2 = 2 * rs;
    const size_t smem_regen = static_cast<size_t>(TR) * rs2 * sizeof(float);
    require(smem_regen <= 200 * 1024, "nbins too large for the beam-search kernels");
    float var_in = 1.0f;  // the initial folds' variance (0 + var_add)
    for (uint32_t st = 0; st < S; ++st) {
        const uint64_t nt = st_trans[st + 1] - st_trans[st];
        const uint32_t nb = static_cast<uint32_t>(st_beam[st + 1] - st_beam[st]);
        const int cur = static_cast<int>(st % 2);
        if (st == 0) {
            a.prev_pool = m_init_pool.as<float>();
            a.prev_counts = m_init_counts.as<uint32_t>();
            a.prev_states = m_init_state.as<lk_dts_state>();
        } else {
            a.prev_pool = m_pool[1 - cur].as<float>();
            a.prev_counts = m_counts[1 - cur].as<uint32_t>();
            a.prev_states = m_states_dev.as<lk_dts_state>() + static_cast<uint64_t>(st - 1) * ncell;
        }
        a.next_pool = m_pool[cur].as<float>();
        a.next_counts = m_counts[cur].as<uint32_t>();
        a.states = m_states_dev.as<lk_dts_state>() + static_cast<uint64_t>(st) * ncell;
        a.trans = m_trans.as<DtsTrans>() + st_trans[st];
        a.beam = m_beam_dev.as<uint32_t>() + st_beam[st];
        a.toff = m_toff.as<uint32_t>() + st_toff[st];
        a.nbeam = nb;
        a.nsurv = m_nsurv.as<uint32_t>() + 2 * st_trans[st];
        a.winner = m_winner.as<int32_t>();
        a.nbranches = m_branching[st];
        a.stage_code = st + 1;
        const float var_new = var_in + 1.0f;
        a.stdnoise = std::sqrt(var_new);
        LK_CUDA(cudaMemsetAsync(m_winner.ptr, 0xFF, m_winner.bytes, s));
        if (nt > 0) {
            const dim3 grid((m_ntrials + T - 1) / T, static_cast<unsigned>(nt), 2);
            if (masked) {
                sc::dispatch_nb_wm(m_nbins, mp, [&](auto nbc, auto wmc) {
                    auto kern = dts_count_kernel<8, decltype(nbc)::value, decltype(wmc)::value>;
                    sc::set_smem(kern, smem_count);
                    kern<<<grid, T, smem_count, s>>>(a, rs, m_sp, mp);
                });
            } else {
                sc::dispatch_nw_nb(m_sp.nwidths, m_nbins, [&](auto nw, auto nbc) {
                    auto kern = dts_count_kernel<decltype(nw)::value, decltype(nbc)::value, 0>;
                    sc::set_smem(kern, smem_count);
                    kern<<<grid, T, smem_count, s>>>(a, rs, m_sp, mp);
                });
            }
            LK_CUDA(cudaGetLastError());
            dts_select_kernel<<<(nb + 127) / 128, 128, 0, s>>>(a);
            LK_CUDA(cudaGetLastError());
        }
        if (masked) {
            sc::dispatch_nb_wm(m_nbins, mp, [&](auto nbc, auto wmc) {
                auto kern = dts_regen_kernel<8, decltype(nbc)::value, decltype(wmc)::value>;
                sc::set_smem(kern, smem_regen);
                kern<<<dim3(static_cast<unsigned>(ncell), 2), TR, smem_regen, s>>>(a, rs2, m_sp, mp);
            });
        } else {
            sc::dispatch_nw_nb(m_sp.nwidths, m_nbins, [&](auto nw, auto nbc) {
                auto kern = dts_regen_kernel<decltype(nw)::value, decltype(nbc)::value, 0>;
                sc::set_smem(kern, smem_regen);
                kern<<<dim3(static_cast<unsigned>(ncell), 2), TR, smem_regen, s>>>(a, rs2, m_sp, mp);
            });
        }
        LK_CUDA(cudaGetLastError());
        var_in = var_new;
    }
    m_states.resize(static_cast<size_t>(S) * ncell);
    LK_CUDA(cudaMemcpyAsync(m_states.data(), m_states_dev.ptr, m_states.size() * sizeof(lk_dts_state),
                            cudaMemcpyDeviceToHost, s));
    uint32_t status = 0;
    LK_CUDA(cudaMemcpyAsync(&status, m_status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    unsigned long long work = 0;
    LK_CUDA(cudaMemcpyAsync(&work, m_work.ptr, sizeof(work), cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    m_transitions = work;
    if (status & kStatusTally) {
        fail(LK_ERR_INTERNAL, "beam search: rebuilt survivors differ from the counted ones");
    }
}

// detail::get_best_path_thresholds (lib/scheme.cpp:98-170).
std::vector<float> DtsExec::best_path(float min_pd) const {
    const uint32_t S = nstages(), NT = nthresholds(), NP = nprobs();
    require(!m_states.empty(), "get_best_path_thresholds: run the scheme first");
    const uint64_t last = static_cast<uint64_t>(S - 1) * NT * NP;
    const lk_dts_state* best = nullptr;
    float best_cost = std::numeric_limits<float>::max();
    for (uint64_t i = 0; i < static_cast<uint64_t>(NT) * NP; ++i) {
        const lk_dts_state& s = m_states[last + i];
        if (s.is_empty != 0 || s.success_h1_cumul < min_pd) {
            continue;
        }
        if (s.cost < best_cost) {
            best_cost = s.cost;
            best = &s;
        }
    }
    if (best == nullptr) {
        return {};
    }
    std::vector<const lk_dts_state*> backward{best};
    float prev_threshold = best->threshold_prev;
    float prev_h1 = best->success_h1_cumul_prev;
    for (uint32_t k = 0; k + 1 < S; ++k) {
        const uint32_t istage = S - 2 - k;
        // utils::find_nearest_index: first index of the smallest |t - value|
        uint32_t ithres = 0;
        float bd = std::fabs(m_thresholds[0] - prev_threshold);
        for (uint32_t i = 1; i < NT; ++i) {
            const float dd = std::fabs(m_thresholds[i] - prev_threshold);
            if (dd < bd) {
                bd = dd;
                ithres = i;
            }
        }
        const int64_t iprob = dts_lower_bin(m_probs, prev_h1);
        require(iprob >= 0 && iprob < static_cast<int64_t>(NP), "probability bin index out of range");
        const lk_dts_state& ps = m_states[static_cast<uint64_t>(istage) * NT * NP +
                                          static_cast<uint64_t>(ithres) * NP +
                                          static_cast<uint64_t>(iprob)];
        if (ps.is_empty != 0) {
            fail(LK_ERR_INTERNAL, "get_best_path_thresholds: backtracking failed (empty state) at stage " +
                                      std::to_string(istage));
        }
        backward.push_back(&ps);
        prev_threshold = ps.threshold_prev;
        prev_h1 = ps.success_h1_cumul_prev;
    }
    std::vector<float> out;
    for (auto it = backward.rbegin(); it != backward.rend(); ++it) {
        out.push_back((*it)->threshold);
    }
    return out;
}

}  // namespace lk
