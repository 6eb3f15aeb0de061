// Monte-Carlo threshold stage on the GPU: one fused pass that builds every
// trial's next-stage fold, scores it and counts it against a threshold grid,
// then the ordered compaction of the trials above the pruning threshold.
//
// Reference: simulate_score_prune_fused (lib/thresholds.cpp:358-431) with
// detection::snr_boxcar_threshold_with_cache (lib/score.cpp:434-462):
//   out_i   = (in[src_i] + noise_i) + signal * scale      (FP32, this order)
//   S/N_w   = ((h_w + b_w) * dmax_w - b_w * sum) / sqrt(var_in + var_add)
//   survive = S/N_w > threshold for some w  (= max_w S/N_w > threshold)
// The noise is drawn on the host (the reference's generator is seeded from
// std::random_device, so its draws are not reproducible) and passed in, so
// the device and the CPU oracle see the same numbers; survivors keep the
// reference's trial order.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <limits>
#include <type_traits>

#include "lk_device.cuh"
#include "lk_mc.hpp"
#include "lk_score.cuh"

namespace lk {

namespace {

constexpr uint32_t kWarp = 32;

struct McArgs {
    const float* in;
    const uint32_t* src;      // NULL: trial i reads input row i
    const float* noise;
    const float* signal;
    const uint32_t* rowmap;   // NULL: noise / per-trial signal row of trial i is i
    uint64_t n;
    uint64_t n_in;            // rows in `in`
    uint64_t n_rows;          // rows in `noise` (and in `signal` when per_trial)
    uint32_t nbins;
    uint32_t* status;         // bad-index flag
    int per_trial;
    float scale;
    float stdnoise;
    const float* thr;         // threshold grid (device), n_thr entries
    uint32_t n_thr;
    const uint8_t* cls;       // optional: class flag of each noise row
    float* max_snr;
    unsigned long long* counts;
    int thr_sorted;           // grid non-decreasing: counted by rank (below)
    float* stage_folds;       // every trial's fold [n][nbins], for the survivors' copy
};

// Input row and noise row of trial i; an index outside its buffer is
// replaced by row 0 and flagged (the entry point then reports an error).
struct TrialRows {
    uint64_t in, noise;
};
__device__ __forceinline__ TrialRows trial_rows(const McArgs& a, uint64_t i, bool flag) {
    uint64_t s = a.src != nullptr ? a.src[i] : i;
    uint64_t rw = a.rowmap != nullptr ? a.rowmap[i] : i;
    if (s >= a.n_in || rw >= a.n_rows) {
        if (flag) {
            atomicOr(a.status, dev::kStatusBadTable);
        }
        s = s >= a.n_in ? 0 : s;
        rw = rw >= a.n_rows ? 0 : rw;
    }
    return {s, rw};
}

__device__ __forceinline__ float stage_value(const McArgs& a, TrialRows t, uint32_t j) {
    const float* sg = a.signal + (a.per_trial ? t.noise * a.nbins : 0);
    return __fadd_rn(__fadd_rn(__ldg(a.in + t.in * a.nbins + j), __ldg(a.noise + t.noise * a.nbins + j)),
                     __fmul_rn(__ldg(sg + j), a.scale));
}

// Trial i's maximum S/N m: stored, and counted against the grid into the
// block's shared counters (see mc_score_kernel).
__device__ __forceinline__ void mc_count(const McArgs& a, uint64_t i, float m, unsigned int* s_cnt,
                                         unsigned int* s_hist2) {
    a.max_snr[i] = m;
    const bool flagged = a.cls != nullptr && a.cls[trial_rows(a, i, false).noise] != 0;
    if (a.thr_sorted) {
        // non-decreasing grid: m > thr[k] exactly for k < r, r the number
        // of grid values below m, so one histogram entry per trial
        // replaces up to n_thr counter increments
        uint32_t r = 0;
        for (uint32_t k = 0; k < a.n_thr; ++k) {
            r += m > a.thr[k] ? 1u : 0u;
        }
        atomicAdd(&s_cnt[r], 1u);
        if (flagged) {
            atomicAdd(&s_hist2[r], 1u);
        }
    } else {
        for (uint32_t k = 0; k < a.n_thr; ++k) {
            if (m > a.thr[k]) {
                atomicAdd(&s_cnt[k], 1u);
                if (flagged) {
                    atomicAdd(&s_cnt[a.n_thr + k], 1u);
                }
            }
        }
    }
}

// The block's counters into the global counts (after a block barrier).
__device__ __forceinline__ void mc_flush(const McArgs& a, const unsigned int* s_cnt,
                                         const unsigned int* s_hist2) {
    const uint32_t T = blockDim.x;
    if (a.thr_sorted) {
        // histogram of ranks -> counts: count[k] = trials of rank > k
        for (uint32_t k = threadIdx.x; k < a.n_thr; k += T) {
            unsigned int c1 = 0, c2 = 0;
            for (uint32_t r = k + 1; r <= a.n_thr; ++r) {
                c1 += s_cnt[r];
                c2 += s_hist2[r];
            }
            if (c1 != 0) {
                atomicAdd(&a.counts[k], static_cast<unsigned long long>(c1));
            }
            if (a.cls != nullptr && c2 != 0) {
                atomicAdd(&a.counts[a.n_thr + k], static_cast<unsigned long long>(c2));
            }
        }
        return;
    }
    const uint32_t ncnt = a.cls != nullptr ? 2 * a.n_thr : a.n_thr;
    for (uint32_t k = threadIdx.x; k < ncnt; k += T) {
        if (s_cnt[k] != 0) {
            atomicAdd(&a.counts[k], static_cast<unsigned long long>(s_cnt[k]));
        }
    }
}

// Block of T trials: warps build the folds in shared memory (lanes over
// bins), then one thread per trial scores its fold; the block's threshold
// counts are summed in shared memory and added to the global counts once.
template <int NW, int NB>
__global__ void mc_score_kernel(McArgs a, uint32_t rs, ScoreParams sp) {
    extern __shared__ float rows[];
    // counts per grid value (or, sorted grid, per rank 0 .. n_thr), all
    // trials then the class-flagged ones
    __shared__ unsigned int s_cnt[2 * LK_MC_MAX_THRESHOLDS + 2];
    unsigned int* s_hist2 = s_cnt + LK_MC_MAX_THRESHOLDS + 1;
    const uint32_t T = blockDim.x;
    const uint64_t p0 = static_cast<uint64_t>(blockIdx.x) * T;
    const uint32_t nhere = static_cast<uint32_t>((a.n - p0) < T ? (a.n - p0) : T);
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    for (uint32_t k = threadIdx.x; k < 2 * LK_MC_MAX_THRESHOLDS + 2; k += T) {
        s_cnt[k] = 0;
    }
#pragma unroll 2
    for (uint32_t p = warp; p < nhere; p += T / kWarp) {
        float* dst = rows + static_cast<size_t>(p) * rs;
        float* keep = a.stage_folds + (p0 + p) * a.nbins;
        const TrialRows tr = trial_rows(a, p0 + p, lane == 0);
        for (uint32_t j = lane; j < a.nbins; j += kWarp) {
            const float x = stage_value(a, tr, j);
            dst[j] = x;
            keep[j] = x;
        }
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const float m = sc::max_snr_div_any<NB, NW>(rows + static_cast<size_t>(threadIdx.x) * rs,
                                                    a.nbins, a.stdnoise, sp);
        mc_count(a, p0 + threadIdx.x, m, s_cnt, s_hist2);
    }
    __syncthreads();
    mc_flush(a, s_cnt, s_hist2);
}

template <int NB, int WM, uint64_t FM>
__global__ void __launch_bounds__(128) mc_score_wm_kernel(McArgs a, MaskScoreParams mp) {
    constexpr int RS = NB + WM + 2;
    extern __shared__ float rows[];
    __shared__ unsigned int s_cnt[2 * LK_MC_MAX_THRESHOLDS + 2];
    unsigned int* s_hist2 = s_cnt + LK_MC_MAX_THRESHOLDS + 1;
    const uint32_t T = blockDim.x;
    const uint64_t p0 = static_cast<uint64_t>(blockIdx.x) * T;
    const uint32_t nhere = static_cast<uint32_t>((a.n - p0) < T ? (a.n - p0) : T);
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    for (uint32_t k = threadIdx.x; k < 2 * LK_MC_MAX_THRESHOLDS + 2; k += T) {
        s_cnt[k] = 0;
    }
    // Phase 1: a warp takes PB trials at a time, lanes over bins; lane q
    // looks up trial q's rows, then every row load of the PB trials is in
    // flight before the first value is formed.
    constexpr int NJ = NB / kWarp;  // bins per lane
    constexpr int PB = NB == 128 ? 4 : 8;
    for (uint32_t pw = warp * PB; pw < nhere; pw += (T / kWarp) * PB) {
        TrialRows mine{0, 0};
        if (lane < static_cast<uint32_t>(PB) && pw + lane < nhere) {
            mine = trial_rows(a, p0 + pw + lane, true);
        }
        float xin[PB][NJ], xnz[PB][NJ], xsg[PB][NJ];
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            const uint64_t rin = __shfl_sync(0xffffffffu, mine.in, q);
            const uint64_t rnz = __shfl_sync(0xffffffffu, mine.noise, q);
            const float* sg = a.signal + (a.per_trial ? rnz * NB : 0);
#pragma unroll
            for (int u = 0; u < NJ; ++u) {
                const uint32_t j = lane + kWarp * u;
                // rows of trials past nhere are row 0 of each buffer (in range, unused)
                xin[q][u] = __ldg(a.in + rin * NB + j);
                xnz[q][u] = __ldg(a.noise + rnz * NB + j);
                xsg[q][u] = __ldg(sg + j);
            }
        }
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            if (pw + q < nhere) {
                float* dst = rows + static_cast<size_t>(pw + q) * RS;
                float* keep = a.stage_folds + (p0 + pw + q) * NB;
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    // (in + noise) + signal * scale, the reference's order
                    const float x = __fadd_rn(__fadd_rn(xin[q][u], xnz[q][u]), __fmul_rn(xsg[q][u], a.scale));
                    dst[lane + kWarp * u] = x;
                    keep[lane + kWarp * u] = x;
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const float best = sc::max_snr_div_wm<NB, WM, FM>(rows + static_cast<size_t>(threadIdx.x) * RS, mp,
                                                      a.stdnoise);
        mc_count(a, p0 + threadIdx.x, best, s_cnt, s_hist2);
    }
    __syncthreads();
    mc_flush(a, s_cnt, s_hist2);
}

// Survivor k (trial idx[k], k < *d_count): its fold, kept by the score
// kernel, copied into out[k], and its noise row recorded. A group of G
// threads per survivor, float4 copies when nbins is a multiple of 4.
__global__ void mc_gather_kernel(McArgs a, const uint32_t* __restrict__ idx,
                                 const uint64_t* __restrict__ d_count, float* __restrict__ out,
                                 uint32_t* __restrict__ ids_out) {
    const uint64_t n = *d_count;
    const uint32_t nb = a.nbins;
    const bool vec = (nb % 4) == 0;
    const uint32_t per_row = vec ? nb / 4 : nb;                // items of one row
    const uint32_t G = per_row >= 32 ? 32 : (per_row >= 16 ? 16 : 8);  // threads per row
    const uint64_t groups = static_cast<uint64_t>(gridDim.x) * (blockDim.x / G);
    const uint32_t sub = threadIdx.x % G;
    for (uint64_t k = blockIdx.x * (blockDim.x / G) + threadIdx.x / G; k < n; k += groups) {
        const uint64_t i = idx[k];
        const float* src = a.stage_folds + i * nb;
        float* dst = out + k * nb;
        if (vec) {
            for (uint32_t q = sub; q < per_row; q += G) {
                reinterpret_cast<float4*>(dst)[q] = __ldg(reinterpret_cast<const float4*>(src) + q);
            }
        } else {
            for (uint32_t q = sub; q < per_row; q += G) {
                dst[q] = __ldg(src + q);
            }
        }
        if (sub == 0 && ids_out != nullptr) {
            ids_out[k] = static_cast<uint32_t>(trial_rows(a, i, false).noise);
        }
    }
}

}  // namespace

McExec::McExec(uint64_t max_trials, uint32_t nbins, const uint32_t* widths, uint32_t nwidths,
               int device)
    : m_max(max_trials), m_nbins(nbins), m_device(device) {
    require(max_trials >= 1 && max_trials <= 0xffffffffULL, "max_trials must lie in [1, 2^32)");
    m_sp = make_score_params(widths, nwidths, nbins);
    DeviceGuard g(device);
    m_max_snr.alloc(max_trials * sizeof(float));
    m_idx.alloc(max_trials * sizeof(uint32_t));
    m_vals.alloc(max_trials * sizeof(float));
    m_scratch.alloc(compact_scratch_bytes(max_trials));
    m_stage_folds.alloc(max_trials * nbins * sizeof(float));
    m_thr.alloc(LK_MC_MAX_THRESHOLDS * sizeof(float));
    m_status.alloc(sizeof(uint32_t));
    LK_CUDA(cudaMemset(m_status.ptr, 0, sizeof(uint32_t)));
}

uint32_t McExec::read_status(cudaStream_t s) {
    DeviceGuard g(m_device);
    uint32_t v = 0;
    LK_CUDA(cudaMemcpyAsync(&v, m_status.ptr, sizeof(v), cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    LK_CUDA(cudaMemsetAsync(m_status.ptr, 0, sizeof(uint32_t), s));
    return v;
}

uint64_t McExec::device_bytes() const {
    return m_max_snr.bytes + m_idx.bytes + m_vals.bytes + m_scratch.bytes + m_thr.bytes + m_stage_folds.bytes +
           m_status.bytes;
}

void McExec::stage(const McStage& st, cudaStream_t s) {
    require(st.ntrials <= m_max, "ntrials exceeds the executor's max_trials");
    require(st.ntrials == 0 || (st.ntrials_in > 0 && st.nrows > 0),
            "ntrials_in and nrows must be positive");
    require(st.n_thr <= LK_MC_MAX_THRESHOLDS, "at most 64 thresholds in the grid");
    require(st.n_thr == 0 || st.thresholds != nullptr, "thresholds must not be NULL");
    require(!(st.var_in + st.var_add < 0.0f), "var_in + var_add must not be negative");
    DeviceGuard g(m_device);
    if (st.n_thr > 0) {
        const uint32_t ncnt = st.d_class != nullptr ? 2 * st.n_thr : st.n_thr;
        LK_CUDA(cudaMemsetAsync(st.d_counts, 0, ncnt * sizeof(uint64_t), s));
        LK_CUDA(cudaMemcpyAsync(m_thr.ptr, st.thresholds, st.n_thr * sizeof(float),
                                cudaMemcpyHostToDevice, s));
    }
    if (st.ntrials == 0) {
        LK_CUDA(cudaMemsetAsync(st.d_count, 0, sizeof(uint64_t), s));
        return;
    }
    McArgs a{};
    a.in = st.d_folds_in;
    a.src = st.d_src;
    a.noise = st.d_noise;
    a.signal = st.d_signal;
    a.rowmap = st.d_rowmap;
    a.n = st.ntrials;
    a.n_in = st.ntrials_in;
    a.n_rows = st.nrows;
    a.nbins = m_nbins;
    a.status = m_status.as<uint32_t>();
    a.per_trial = st.signal_per_trial ? 1 : 0;
    a.scale = st.signal_scale;
    a.stdnoise = std::sqrt(st.var_in + st.var_add);  // float, as sqrt(var_new) in the reference
    a.thr = m_thr.as<float>();
    a.n_thr = st.n_thr;
    // the rank count needs {k : m > thr[k]} to be a prefix for every m: a
    // non-decreasing grid without NaN
    a.thr_sorted = std::is_sorted(st.thresholds, st.thresholds + st.n_thr) &&
                           std::none_of(st.thresholds, st.thresholds + st.n_thr,
                                        [](float x) { return std::isnan(x); })
                       ? 1
                       : 0;
    a.cls = st.d_class;
    a.max_snr = st.d_max_snr != nullptr ? st.d_max_snr : m_max_snr.as<float>();
    a.stage_folds = m_stage_folds.as<float>();
    a.counts = reinterpret_cast<unsigned long long*>(st.d_counts);
    const uint32_t rs = sc::row_stride(m_nbins, m_sp.wmax);
    const uint32_t T = sc::profiles_per_block(rs);
    const size_t smem = static_cast<size_t>(T) * rs * sizeof(float);
    const uint64_t blocks = (st.ntrials + T - 1) / T;
    require(blocks <= 0x7fffffffULL, "too many trials");
    auto launch = [&](auto kern) {
        sc::set_smem(kern, smem);
        kern<<<static_cast<unsigned>(blocks), T, smem, s>>>(a, rs, m_sp);
    };
    MaskScoreParams mp{};
    if (make_mask_score_params(m_sp, m_nbins, &mp)) {
        // the mask path: nbins 32 / 64 / 128, strictly increasing widths <= 32
        sc::dispatch_nb_wm(m_nbins, mp, [&](auto nbc, auto wmc) {
            constexpr int NB = decltype(nbc)::value;
            constexpr int WM = decltype(wmc)::value;
            auto kern = mc_score_wm_kernel<NB, WM, 0>;
            if constexpr (WM == 16) {
                if (mp.wmask == sc::kFixedMask16 && mp.wmax == 16) {
                    kern = mc_score_wm_kernel<NB, WM, sc::kFixedMask16>;
                }
            }
            const uint32_t Tw = 128;
            const size_t smem_w = static_cast<size_t>(Tw) * (NB + WM + 2) * sizeof(float);
            sc::set_smem(kern, smem_w);
            const uint64_t bw = (st.ntrials + Tw - 1) / Tw;
            kern<<<static_cast<unsigned>(bw), Tw, smem_w, s>>>(a, mp);
        });
    } else {
        sc::dispatch_nw_nb(m_sp.nwidths, m_nbins, [&](auto nw, auto nbc) {
            launch(mc_score_kernel<decltype(nw)::value, decltype(nbc)::value>);
        });
    }
    LK_CUDA(cudaGetLastError());
    // S/N > threshold  <=>  S/N >= the next float above the threshold.
    const float thr_ge = std::nextafter(st.threshold, std::numeric_limits<float>::infinity());
    compact_ge(a.max_snr, st.ntrials, thr_ge, m_idx.as<uint32_t>(), m_vals.as<float>(),
               st.ntrials, st.d_count, m_scratch.ptr, s);
    const uint64_t gblocks = std::min<uint64_t>((st.ntrials + 7) / 8, 148 * 16);
    mc_gather_kernel<<<static_cast<unsigned>(gblocks), 256, 0, s>>>(
        a, m_idx.as<uint32_t>(), st.d_count, st.d_folds_out, st.d_ids_out);
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
