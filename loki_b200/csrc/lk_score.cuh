// Boxcar scoring helpers shared by the FFA scorer (score.cu) and the pruning
// leaf kernel (prune.cu). Reference: snr_boxcar_impl (lib/score.cpp:95-172),
// score_and_filter_max_with_cache (lib/score.cpp:213-259), circular_prefix_sum
// and diff_max (lib/utils.cpp:22-67).
#pragma once

#include <cfloat>
#include <cstdint>
#include <type_traits>

#include "lk_internal.hpp"
#include "lk_kernels.hpp"

namespace lk::sc {

// Odd row stride holding a profile and its circular extension.
inline uint32_t row_stride(uint32_t nbins, uint32_t wmax) { return (nbins + wmax) | 1u; }

__device__ __forceinline__ float normalise(float e, float v) {
    // 1.0F / std::sqrt(v) then e * that (lib/score.cpp:134-136): both
    // correctly rounded, so rcp_rn(sqrt_rn(v)) == 1.0F / sqrt(v) exactly.
    return __fmul_rn(e, __frcp_rn(__fsqrt_rn(v)));
}

// Scores the normalised profile staged at r (in place) and returns the
// largest S/N over the widths. NW >= sp.nwidths is the compile-time width
// capacity (8, 16 or 32): the width loops are unrolled to NW, so a small NW
// avoids evaluating unused width slots.
template <int NW>
__device__ __forceinline__ float score_row(float* r, uint32_t nbins, float inv_stdnoise,
                                           const ScoreParams& sp, int mode, float* out) {
    float acc = r[0];
    for (uint32_t j = 1; j < nbins; ++j) {
        acc = __fadd_rn(acc, r[j]);
        r[j] = acc;
    }
    const float sum = acc;
    for (uint32_t k = 0; k < sp.wmax; ++k) {
        r[nbins + k] = __fadd_rn(r[k], sum);
    }
    float dm[NW];
#pragma unroll
    for (int iw = 0; iw < NW; ++iw) {
        dm[iw] = -FLT_MAX;
    }
    for (uint32_t i = 0; i < nbins; ++i) {
        const float ri = r[i];
#pragma unroll
        for (int iw = 0; iw < NW; ++iw) {
            if (iw < static_cast<int>(sp.nwidths)) {
                const float d = __fsub_rn(r[i + sp.widths[iw]], ri);
                dm[iw] = (dm[iw] < d) ? d : dm[iw];
            }
        }
    }
    float best = -FLT_MAX;
#pragma unroll
    for (int iw = 0; iw < NW; ++iw) {
        if (iw < static_cast<int>(sp.nwidths)) {
            const float base = __fsub_rn(__fmul_rn(sp.hb[iw], dm[iw]), __fmul_rn(sp.b[iw], sum));
            const float snr = __fmul_rn(base, inv_stdnoise);
            if (mode == LK_SCORE_PER_WIDTH) {
                out[iw] = snr;
            }
            best = (best < snr) ? snr : best;
        }
    }
    if (mode == LK_SCORE_MAX) {
        out[0] = best;
    }
    return best;
}

// Largest S/N of the (raw, 2-D) profile staged at r with every width's S/N
// divided by stdnoise, as detection::snr_boxcar_threshold_with_cache does
// (lib/score.cpp:434-462). Prefix sums are written in place.
template <int NW>
__device__ __forceinline__ float max_snr_div(float* r, uint32_t nbins, float stdnoise,
                                             const ScoreParams& sp) {
    float acc = r[0];
    for (uint32_t j = 1; j < nbins; ++j) {
        acc = __fadd_rn(acc, r[j]);
        r[j] = acc;
    }
    const float sum = acc;
    for (uint32_t k = 0; k < sp.wmax; ++k) {
        r[nbins + k] = __fadd_rn(r[k], sum);
    }
    float dm[NW];
#pragma unroll
    for (int iw = 0; iw < NW; ++iw) {
        dm[iw] = -FLT_MAX;
    }
    for (uint32_t i = 0; i < nbins; ++i) {
        const float ri = r[i];
#pragma unroll
        for (int iw = 0; iw < NW; ++iw) {
            if (iw < static_cast<int>(sp.nwidths)) {
                const float d = __fsub_rn(r[i + sp.widths[iw]], ri);
                dm[iw] = (dm[iw] < d) ? d : dm[iw];
            }
        }
    }
    float best = -FLT_MAX;
#pragma unroll
    for (int iw = 0; iw < NW; ++iw) {
        if (iw < static_cast<int>(sp.nwidths)) {
            const float base = __fsub_rn(__fmul_rn(sp.hb[iw], dm[iw]), __fmul_rn(sp.b[iw], sum));
            const float snr = __fdiv_rn(base, stdnoise);
            best = (best < snr) ? snr : best;
        }
    }
    return best;
}

// ---- compile-time nbins ------------------------------------------------
// The same operations as score_row / max_snr_div (sequential prefix sum,
// circular extension, window differences, maxima), with nbins a template
// constant so every loop over bins unrolls and each shared-memory access is
// one load with an immediate offset. Width slots at or beyond sp.nwidths
// repeat width 0 and are ignored, so no slot needs a predicate.

template <int NB, int NW>
__device__ __forceinline__ float prefix_dmax_nb(float* r, const ScoreParams& sp, float (&dm)[NW]) {
    float acc = r[0];
#pragma unroll
    for (int j = 1; j < NB; ++j) {
        acc = __fadd_rn(acc, r[j]);
        r[j] = acc;
    }
    const float sum = acc;
    for (uint32_t k = 0; k < sp.wmax; ++k) {
        r[NB + k] = __fadd_rn(r[k], sum);
    }
    const float* base[NW];
#pragma unroll
    for (int iw = 0; iw < NW; ++iw) {
        base[iw] = r + (iw < static_cast<int>(sp.nwidths) ? sp.widths[iw] : sp.widths[0]);
        dm[iw] = -FLT_MAX;
    }
#pragma unroll
    for (int i = 0; i < NB; ++i) {
        const float ri = r[i];
#pragma unroll
        for (int iw = 0; iw < NW; ++iw) {
            const float d = __fsub_rn(base[iw][i], ri);
            dm[iw] = (dm[iw] < d) ? d : dm[iw];
        }
    }
    return sum;
}

template <int NB, int NW>
__device__ __forceinline__ float score_row_nb(float* r, float inv_stdnoise, const ScoreParams& sp,
                                              int mode, float* out) {
    float dm[NW];
    const float sum = prefix_dmax_nb<NB, NW>(r, sp, dm);
    float best = -FLT_MAX;
#pragma unroll
    for (int iw = 0; iw < NW; ++iw) {
        if (iw < static_cast<int>(sp.nwidths)) {
            const float base = __fsub_rn(__fmul_rn(sp.hb[iw], dm[iw]), __fmul_rn(sp.b[iw], sum));
            const float snr = __fmul_rn(base, inv_stdnoise);
            if (mode == LK_SCORE_PER_WIDTH) {
                out[iw] = snr;
            }
            best = (best < snr) ? snr : best;
        }
    }
    if (mode == LK_SCORE_MAX) {
        out[0] = best;
    }
    return best;
}

template <int NB, int NW>
__device__ __forceinline__ float max_snr_div_nb(float* r, float stdnoise, const ScoreParams& sp) {
    float dm[NW];
    const float sum = prefix_dmax_nb<NB, NW>(r, sp, dm);
    float best = -FLT_MAX;
#pragma unroll
    for (int iw = 0; iw < NW; ++iw) {
        if (iw < static_cast<int>(sp.nwidths)) {
            const float base = __fsub_rn(__fmul_rn(sp.hb[iw], dm[iw]), __fmul_rn(sp.b[iw], sum));
            const float snr = __fdiv_rn(base, stdnoise);
            best = (best < snr) ? snr : best;
        }
    }
    return best;
}

// ---- masked widths (nbins 32 / 64 / 128, strictly increasing widths <= 32) --

// Three-input max.f32 (sm_100): the largest non-NaN input, as two nested fmaxf.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Exact reference maximum (first maximum kept) of p[i + w] - p[i].
__device__ __noinline__ inline float dmax_first(const float* r, uint32_t w, uint32_t nbins) {
    float m = -FLT_MAX;
    for (uint32_t i = 0; i < nbins; ++i) {
        const float d = __fsub_rn(r[i + w], r[i]);
        m = (m < d) ? d : m;
    }
    return m;
}

// max_snr_div for a profile of NB bins at r (8-byte aligned, room for NB +
// WM + 2 floats; prefix sums written in place) and the width mask mp: the
// same IEEE operations -- sequential prefix, circular extension, window
// differences, ((h + b) dmax - b sum) / stdnoise per width, the maximum over
// widths in width order -- with the row read two bins per 64-bit access,
// windows of 16 positions in registers, every width a compile-time offset
// taken when its mask bit is set, and each width's maximum by a tree of
// three-input maxima (equal in value to the reference's scan; a zero
// maximum, whose sign the tree may not keep, is recomputed with its rule).
// FM: the width mask as a compile-time constant (mp.wmask == FM; its widest
// width WM), so that the width bodies not taken are not generated, or 0 to
// test mp.wmask at run time.
// out: when given, each width's S/N is also stored at out[slot of the width].
template <int NB, int WM, uint64_t FM = 0>
__device__ __forceinline__ float max_snr_div_wm(float* r, const MaskScoreParams& mp, float stdnoise,
                                                float* out = nullptr) {
    constexpr int CH = 16;
    static_assert(NB % CH == 0 && WM <= 32, "masked scorer shape");
    float2* r2 = reinterpret_cast<float2*>(r);
    float acc = 0.0f;
#pragma unroll
    for (int j = 0; j < NB / 2; ++j) {
        const float2 x = r2[j];
        const float a0 = j == 0 ? x.x : __fadd_rn(acc, x.x);
        acc = __fadd_rn(a0, x.y);
        r2[j] = make_float2(a0, acc);
    }
    const float sum = acc;
    auto taken = [&](int w) -> bool {
        return FM != 0 ? ((FM >> w) & 1ull) != 0 : ((mp.wmask >> w) & 1ull) != 0;
    };
    if constexpr (FM != 0) {
        static_assert((FM >> (WM + 1)) == 0 && ((FM >> WM) & 1ull), "fixed mask's widest width is WM");
#pragma unroll
        for (int k = 0; k < WM; ++k) {
            r[NB + k] = __fadd_rn(r[k], sum);
        }
    } else {
        for (uint32_t k = 0; k < mp.wmax; ++k) {
            r[NB + k] = __fadd_rn(r[k], sum);
        }
    }
    float dm[WM + 1];
#pragma unroll
    for (int w = 1; w <= WM; ++w) {
        dm[w] = -FLT_MAX;
    }
#pragma unroll 1
    for (int c = 0; c < NB; c += CH) {
        float win[CH + WM];
#pragma unroll
        for (int k = 0; k < (CH + WM) / 2; ++k) {
            const float2 x = r2[c / 2 + k];
            win[2 * k] = x.x;
            win[2 * k + 1] = x.y;
        }
#pragma unroll
        for (int w = 1; w <= WM; ++w) {
            if (taken(w)) {
                float d[CH];
#pragma unroll
                for (int k = 0; k < CH; ++k) {
                    d[k] = __fsub_rn(win[k + w], win[k]);
                }
                const float m0 = fmax3(d[0], d[1], d[2]);
                const float m1 = fmax3(d[3], d[4], d[5]);
                const float m2 = fmax3(d[6], d[7], d[8]);
                const float m3 = fmax3(d[9], d[10], d[11]);
                const float m4 = fmax3(d[12], d[13], d[14]);
                dm[w] = fmax3(dm[w], fmax3(m0, m1, m2), fmax3(m3, m4, d[15]));
            }
        }
    }
    float best = -FLT_MAX;
#pragma unroll
    for (int w = 1; w <= WM; ++w) {
        if (taken(w)) {
            float d = dm[w];
            if (d == 0.0f) {
                d = dmax_first(r, static_cast<uint32_t>(w), NB);
            }
            const float base = __fsub_rn(__fmul_rn(mp.hb[w], d), __fmul_rn(mp.b[w], sum));
            const float snr = __fdiv_rn(base, stdnoise);
            if (out != nullptr) {
                out[mp.slot[w]] = snr;
            }
            best = (best < snr) ? snr : best;
        }
    }
    return best;
}

// Width mask of the widths {1, 2, 3, 4, 6, 8, 12, 16} (the benchmark widths),
// for the compile-time mask form of the masked scorers.
constexpr uint64_t kFixedMask16 = (1ull << 1) | (1ull << 2) | (1ull << 3) | (1ull << 4) | (1ull << 6) |
                                  (1ull << 8) | (1ull << 12) | (1ull << 16);

// Calls f(NB, WM) for the masked scorer's shape of (nbins, mp) -- NB 32 / 64 /
// 128, WM the width bucket 8 / 16 / 32.
template <class F>
void dispatch_nb_wm(uint32_t nbins, const MaskScoreParams& mp, F&& f) {
    auto by_wm = [&](auto nbc) {
        if (mp.wmax <= 8) {
            f(nbc, std::integral_constant<int, 8>{});
        } else if (mp.wmax <= 16) {
            f(nbc, std::integral_constant<int, 16>{});
        } else {
            f(nbc, std::integral_constant<int, 32>{});
        }
    };
    if (nbins == 32) {
        by_wm(std::integral_constant<int, 32>{});
    } else if (nbins == 64) {
        by_wm(std::integral_constant<int, 64>{});
    } else {
        by_wm(std::integral_constant<int, 128>{});
    }
}

// score_row with nbins dispatched to a compile-time constant when it is NB.
template <int NB, int NW>
__device__ __forceinline__ float score_row_any(float* r, uint32_t nbins, float inv_stdnoise,
                                               const ScoreParams& sp, int mode, float* out) {
    if constexpr (NB > 0) {
        return score_row_nb<NB, NW>(r, inv_stdnoise, sp, mode, out);
    } else {
        return score_row<NW>(r, nbins, inv_stdnoise, sp, mode, out);
    }
}

// Calls f(integral_constant<int, NW>, integral_constant<int, NB>) with NW the
// width capacity (8, 16, 32) and NB = nbins when it is 32, 64 or 128 (and at
// most 16 widths), else NB = 0 (runtime nbins).
template <class F>
void dispatch_nw_nb(uint32_t nwidths, uint32_t nbins, F&& f) {
    auto by_nb = [&](auto nw) {
        constexpr int NW = decltype(nw)::value;
        if constexpr (NW <= 16) {
            if (nbins == 32) {
                f(nw, std::integral_constant<int, 32>{});
                return;
            }
            if (nbins == 64) {
                f(nw, std::integral_constant<int, 64>{});
                return;
            }
            if (nbins == 128) {
                f(nw, std::integral_constant<int, 128>{});
                return;
            }
        }
        f(nw, std::integral_constant<int, 0>{});
    };
    if (nwidths <= 8) {
        by_nb(std::integral_constant<int, 8>{});
    } else if (nwidths <= 16) {
        by_nb(std::integral_constant<int, 16>{});
    } else {
        by_nb(std::integral_constant<int, 32>{});
    }
}

template <int NB, int NW>
__device__ __forceinline__ float max_snr_div_any(float* r, uint32_t nbins, float stdnoise,
                                                 const ScoreParams& sp) {
    if constexpr (NB > 0) {
        return max_snr_div_nb<NB, NW>(r, stdnoise, sp);
    } else {
        return max_snr_div<NW>(r, nbins, stdnoise, sp);
    }
}

// Profiles per block so that the staged rows fit comfortably in shared memory.
inline uint32_t profiles_per_block(uint32_t rs) {
    const size_t per = static_cast<size_t>(rs) * sizeof(float);
    uint32_t T = 128;
    while (T > 32 && T * per > 48 * 1024) {
        T -= 32;
    }
    if (T * per > 200 * 1024) {
        fail(LK_ERR_UNSUPPORTED, "nbins too large for the boxcar scorer");
    }
    return T;
}

template <class K>
void set_smem(K kern, size_t smem) {
    if (smem > 48 * 1024) {
        LK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(smem)));
    }
}

}  // namespace lk::sc
