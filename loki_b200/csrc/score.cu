// Boxcar matched-filter S/N of folded profiles, and the final FFA level
// fused with it.
//
// Per profile (reference: snr_boxcar_impl, lib/score.cpp:95-172;
// circular_prefix_sum / diff_max, lib/utils.cpp:22-67):
//   x_j    = E_j * (1 / sqrt(V_j))            (3-D folds; 2-D folds use x = fold)
//   p      = inclusive prefix sum of x, extended circularly by wmax bins
//   dmax_w = max_i (p[i + w] - p[i]),  i in [0, nbins)
//   snr_w  = ((h_w + b_w) * dmax_w - b_w * p[nbins-1]) * inv_stdnoise
// with h_w = sqrt((n - w) / (n w)), b_w = w h_w / (n - w).
//
// Two phases per block: (1) warps build the normalised profiles x in shared
// memory (lanes over bins: coalesced loads, element-parallel sqrt and
// reciprocal); (2) one thread per profile runs the reference's sequential
// prefix sum and the width maxima. Every operation is IEEE round-to-nearest
// in the reference's order, so scores are bit-identical. Profiles are staged
// with an odd row stride, so the 32 threads of a warp, each at the same column
// of a different row, hit 32 different banks.
#include <cfloat>
#include <cmath>
#include <type_traits>

#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_merge.cuh"
#include "lk_score.cuh"

namespace lk {

namespace {

constexpr int kWarp = 32;
using namespace sc;

template <int NW, int NB>
__global__ void score_kernel(const float* __restrict__ folds, uint64_t nprof, uint32_t nbins,
                             bool is3d, float inv_stdnoise, uint32_t rs, ScoreParams sp, int mode,
                             float* __restrict__ scores) {
    extern __shared__ float rows[];
    const uint32_t T = blockDim.x;
    const uint64_t p0 = static_cast<uint64_t>(blockIdx.x) * T;
    const uint32_t nhere = static_cast<uint32_t>((nprof - p0) < T ? (nprof - p0) : T);
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const uint32_t plen = is3d ? 2 * nbins : nbins;
    for (uint32_t p = warp; p < nhere; p += T / kWarp) {
        const float* src = folds + (p0 + p) * plen;
        float* dst = rows + static_cast<size_t>(p) * rs;
        for (uint32_t j = lane; j < nbins; j += kWarp) {
            dst[j] = is3d ? normalise(__ldg(src + j), __ldg(src + nbins + j)) : __ldg(src + j);
        }
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const uint64_t p = p0 + threadIdx.x;
        const uint32_t nout = mode == LK_SCORE_PER_WIDTH ? sp.nwidths : 1;
        score_row_any<NB, NW>(rows + static_cast<size_t>(threadIdx.x) * rs, nbins, inv_stdnoise, sp,
                              mode, scores + p * nout);
    }
}

// Final FFA level (one output segment) merged and normalised straight into
// shared memory, then scored; the final fold never reaches global memory.
// Block = up to T consecutive frequency cells of one outer row; blocks are
// numbered frequency-tile-major (see merge.cu).
//
// Phase 1 keeps many loads in flight: a warp takes PB profiles at a time,
// loads their coordinates with one lane each, then issues every tail/head
// load of the PB profiles (NJ = ceil(nbins / 32) bins per lane; NJ == 0
// selects a generic loop for large nbins) before the first add.
template <bool TAYLOR, int NW, int NJ, int PB, class TIn, int NB>
__global__ void merge_score_kernel(const TIn* __restrict__ in, const void* __restrict__ coords,
                                   uint32_t n_inner, uint32_t n_outer, uint64_t nprev,
                                   uint32_t nbins, uint32_t rs, ScoreParams sp, int mode,
                                   float* __restrict__ scores, float* __restrict__ cmax) {
    extern __shared__ float rows[];
    // Series of a batch on grid.y: input segments 2b and 2b + 1, scores b.
    in += static_cast<uint64_t>(blockIdx.y) * 2 * nprev * 2 * nbins;
    scores += static_cast<uint64_t>(blockIdx.y) * n_inner * n_outer *
              (mode == LK_SCORE_PER_WIDTH ? sp.nwidths : 1);
    if (cmax != nullptr) {
        cmax += static_cast<uint64_t>(blockIdx.y) * n_inner * n_outer;
    }
    const uint32_t T = blockDim.x;
    const uint32_t tile = blockIdx.x / n_outer;
    const uint32_t outer = blockIdx.x - tile * n_outer;
    const uint32_t j0 = tile * T;
    const uint32_t nhere = min(T, n_inner - j0);
    const uint64_t c0 = static_cast<uint64_t>(outer) * n_inner + j0;
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const uint32_t plen = 2 * nbins;
    const TIn* head_base = in + nprev * plen;  // segment 1 of the previous level
    if constexpr (NJ == 0) {
#pragma unroll 2
        for (uint32_t p = warp; p < nhere; p += T / kWarp) {
            const MergeCoord mc = load_merge_coord<TAYLOR>(coords, c0 + p, nbins);
            const TIn* tail = in + static_cast<uint64_t>(mc.it) * plen;
            const TIn* head = head_base + static_cast<uint64_t>(mc.ih) * plen;
            float* dst = rows + static_cast<size_t>(p) * rs;
            for (uint32_t j = lane; j < nbins; j += kWarp) {
                const uint32_t jt = j >= mc.st ? j - mc.st : j + nbins - mc.st;
                const uint32_t jh = j >= mc.sh ? j - mc.sh : j + nbins - mc.sh;
                const float e = __fadd_rn(dev::Store<TIn>::load(tail + jt),
                                          dev::Store<TIn>::load(head + jh));
                const float v = __fadd_rn(dev::Store<TIn>::load(tail + nbins + jt),
                                          dev::Store<TIn>::load(head + nbins + jh));
                dst[j] = normalise(e, v);
            }
        }
    } else {
        for (uint32_t p0 = warp * PB; p0 < nhere; p0 += (T / kWarp) * PB) {
            MergeCoord mine{0, 0, 0, 0};
            if (lane < PB && p0 + lane < nhere) {
                mine = load_merge_coord<TAYLOR>(coords, c0 + p0 + lane, nbins);
            }
            float te[PB][NJ], tv[PB][NJ], he[PB][NJ], hv[PB][NJ];
#pragma unroll
            for (int q = 0; q < PB; ++q) {
                const uint32_t it = __shfl_sync(0xffffffffu, mine.it, q);
                const uint32_t ih = __shfl_sync(0xffffffffu, mine.ih, q);
                const uint32_t st = __shfl_sync(0xffffffffu, mine.st, q);
                const uint32_t sh = __shfl_sync(0xffffffffu, mine.sh, q);
                const bool live = p0 + q < nhere;
                const TIn* tail = in + static_cast<uint64_t>(it) * plen;
                const TIn* head = head_base + static_cast<uint64_t>(ih) * plen;
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    if constexpr (NB > 0) {
                        // nbins == NB == 32 * NJ: every lane's bins are in range;
                        // rows past nhere read row 0 (in range) and are not used
                        const uint32_t j = lane + 32u * u;
                        const TIn* pt = (live ? tail : in) + ((j - st) & (NB - 1));
                        const TIn* ph = (live ? head : head_base) + ((j - sh) & (NB - 1));
                        te[q][u] = dev::Store<TIn>::load(pt);
                        tv[q][u] = dev::Store<TIn>::load(pt + NB);
                        he[q][u] = dev::Store<TIn>::load(ph);
                        hv[q][u] = dev::Store<TIn>::load(ph + NB);
                    } else {
                        const uint32_t jr = lane + 32u * u;
                        const bool ok = live && jr < nbins;
                        const uint32_t j = ok ? jr : 0u;  // keep every address inside the rows
                        const uint32_t jt = j >= st ? j - st : j + nbins - st;
                        const uint32_t jh = j >= sh ? j - sh : j + nbins - sh;
                        te[q][u] = ok ? dev::Store<TIn>::load(tail + jt) : 0.0f;
                        tv[q][u] = ok ? dev::Store<TIn>::load(tail + nbins + jt) : 1.0f;
                        he[q][u] = ok ? dev::Store<TIn>::load(head + jh) : 0.0f;
                        hv[q][u] = ok ? dev::Store<TIn>::load(head + nbins + jh) : 1.0f;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < PB; ++q) {
                if (p0 + q < nhere) {
                    float* dst = rows + static_cast<size_t>(p0 + q) * rs;
#pragma unroll
                    for (int u = 0; u < NJ; ++u) {
                        const uint32_t j = lane + 32u * u;
                        if (j < nbins) {
                            dst[j] = normalise(__fadd_rn(te[q][u], he[q][u]),
                                               __fadd_rn(tv[q][u], hv[q][u]));
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const uint64_t c = c0 + threadIdx.x;
        const uint32_t nout = mode == LK_SCORE_PER_WIDTH ? sp.nwidths : 1;
        const float best = score_row_any<NB, NW>(rows + static_cast<size_t>(threadIdx.x) * rs,
                                                 nbins, 1.0f, sp, mode, scores + c * nout);
        if (cmax != nullptr) {
            cmax[c] = best;
        }
    }
}

}  // namespace

// First parameter type of a merge_score_kernel instantiation.
template <class K> struct KernelInput;
template <class TIn, class... Rest> struct KernelInput<void (*)(const TIn*, Rest...)> {
    using type = TIn;
};

ScoreParams make_score_params(const uint32_t* widths, uint32_t nwidths, uint32_t nbins) {
    require(nwidths >= 1 && nwidths <= LK_MAX_WIDTHS, "number of widths must be in [1, 32]");
    require(nbins >= 2, "nbins must be at least 2 for scoring");
    ScoreParams sp{};
    sp.nwidths = nwidths;
    sp.wmax = 0;
    for (uint32_t i = 0; i < nwidths; ++i) {
        const uint32_t w = widths[i];
        require(w >= 1 && w < nbins, "score widths must lie in [1, nbins)");
        sp.widths[i] = w;
        sp.wmax = w > sp.wmax ? w : sp.wmax;
        // BoxcarWidthsCache / snr_boxcar_impl (lib/score.cpp:108-116): FP32.
        const float h = std::sqrt(static_cast<float>(nbins - w) / static_cast<float>(nbins * w));
        const float b = static_cast<float>(w) * h / static_cast<float>(nbins - w);
        sp.hb[i] = h + b;
        sp.b[i] = b;
    }
    return sp;
}

void score_folds(const float* d_folds, uint64_t nprof, uint32_t nbins, bool is3d,
                 float inv_stdnoise, const ScoreParams& sp, int mode, float* d_scores,
                 cudaStream_t s) {
    if (nprof == 0) {
        return;
    }
    const uint32_t rs = row_stride(nbins, sp.wmax);
    const uint32_t T = profiles_per_block(rs);
    const size_t smem = static_cast<size_t>(T) * rs * sizeof(float);
    const uint64_t blocks = (nprof + T - 1) / T;
    require(blocks <= 0x7fffffffULL, "too many profiles");
    auto launch = [&](auto kern) {
        set_smem(kern, smem);
        kern<<<static_cast<unsigned>(blocks), T, smem, s>>>(d_folds, nprof, nbins, is3d,
                                                            inv_stdnoise, rs, sp, mode, d_scores);
    };
    dispatch_nw_nb(sp.nwidths, nbins, [&](auto nw, auto nbc) {
        launch(score_kernel<decltype(nw)::value, decltype(nbc)::value>);
    });
    LK_CUDA(cudaGetLastError());
}

void merge_score_level(const void* d_in, const void* d_coords, bool taylor, uint64_t n_inner,
                       uint64_t n_outer, uint64_t ncoords_prev, uint32_t nbins,
                       const ScoreParams& sp, int mode, float* d_scores, cudaStream_t s,
                       uint64_t nbatch, bool in_bf16, float* d_cmax, uint32_t cells_per_block) {
    require(nbatch >= 1 && nbatch <= 65535, "nbatch must lie in [1, 65535]");
    if (n_inner == 0 || n_outer == 0) {
        return;
    }
    const uint32_t rs = row_stride(nbins, sp.wmax);
    // cells per block: a multiple of 32 up to the shared-memory default
    const uint32_t Tmax = profiles_per_block(rs);
    const uint32_t T = (cells_per_block >= 32 && cells_per_block % 32 == 0 && cells_per_block <= Tmax)
                           ? cells_per_block
                           : Tmax;
    const size_t smem = static_cast<size_t>(T) * rs * sizeof(float);
    const uint64_t tiles = (n_inner + T - 1) / T;
    require(tiles * n_outer <= 0x7fffffffULL && n_inner <= 0xffffffffULL,
            "final level too large for the launch grid");
    const auto blocks = static_cast<unsigned>(tiles * n_outer);
    const auto ni = static_cast<uint32_t>(n_inner);
    const auto no = static_cast<uint32_t>(n_outer);
    auto launch = [&](auto kern) {
        set_smem(kern, smem);
        using TIn = typename KernelInput<decltype(kern)>::type;
        kern<<<dim3(blocks, static_cast<unsigned>(nbatch)), T, smem, s>>>(
            static_cast<const TIn*>(d_in), d_coords, ni, no, ncoords_prev, nbins, rs, sp, mode,
            d_scores, d_cmax);
    };
    const int nwb = sp.nwidths <= 8 ? 8 : (sp.nwidths <= 16 ? 16 : 32);
    const int nj = nbins <= 32 ? 1 : (nbins <= 64 ? 2 : (nbins <= 128 ? 4 : (nbins <= 256 ? 8 : 0)));
    // Dispatch (taylor, width bucket, bins per lane); PB * NJ = 16 loads of
    // each kind in flight per lane.
    auto pick = [&](auto tg, auto tin) {
        constexpr bool TG = decltype(tg)::value;
        using TI = decltype(tin);
        // nbins of exactly 32, 64 or 128 (up to 16 widths) score with
        // compile-time nbins.
        const bool fixed = sp.nwidths <= 16 && (nbins == 32 || nbins == 64 || nbins == 128);
        auto by_nj = [&](auto nwc) {
            constexpr int NWC = decltype(nwc)::value;
            constexpr int FX = NWC <= 16 ? 1 : 0;
            if (nj == 1) {
                fixed ? launch(merge_score_kernel<TG, NWC, 1, 16, TI, 32 * FX>)
                      : launch(merge_score_kernel<TG, NWC, 1, 16, TI, 0>);
            } else if (nj == 2) {
                fixed ? launch(merge_score_kernel<TG, NWC, 2, 8, TI, 64 * FX>)
                      : launch(merge_score_kernel<TG, NWC, 2, 8, TI, 0>);
            } else if (nj == 4) {
                fixed ? launch(merge_score_kernel<TG, NWC, 4, 4, TI, 128 * FX>)
                      : launch(merge_score_kernel<TG, NWC, 4, 4, TI, 0>);
            } else if (nj == 8) {
                launch(merge_score_kernel<TG, NWC, 8, 2, TI, 0>);
            } else {
                launch(merge_score_kernel<TG, NWC, 0, 1, TI, 0>);
            }
        };
        if (nwb == 8) by_nj(std::integral_constant<int, 8>{});
        else if (nwb == 16) by_nj(std::integral_constant<int, 16>{});
        else by_nj(std::integral_constant<int, 32>{});
    };
    if (taylor) {
        in_bf16 ? pick(std::true_type{}, __nv_bfloat16{}) : pick(std::true_type{}, float{});
    } else {
        in_bf16 ? pick(std::false_type{}, __nv_bfloat16{}) : pick(std::false_type{}, float{});
    }
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
