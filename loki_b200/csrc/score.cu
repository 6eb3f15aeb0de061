// Boxcar matched-filter S/N of folded profiles, and the final FFA level
// fused with it.
//
// Per profile (reference: snr_boxcar_impl, lib/score.cpp:95-172;
// circular_prefix_sum / diff_max, lib/utils.cpp:22-67):
//   x_j   = E_j * (1 / sqrt(V_j))            (3-D folds; 2-D folds use x = fold)
//   p     = inclusive prefix sum of x, extended circularly by wmax bins
//   dmax_w = max_i (p[i + w] - p[i]),  i in [0, nbins)
//   snr_w = ((h_w + b_w) * dmax_w - b_w * p[nbins-1]) * inv_stdnoise
// with h_w = sqrt((n - w) / (n w)), b_w = w h_w / (n - w).
//
// One thread scores one profile, sequentially, with IEEE-rounded operations
// in the reference's order, so scores are bit-identical to the reference's
// CPU code. Profiles are staged in shared memory with an odd row stride:
// threads of a warp touch the same column of 32 different rows, which falls
// in 32 different banks.
#include <cfloat>
#include <cmath>

#include "lk_device.cuh"
#include "lk_kernels.hpp"

namespace lk {

namespace {


struct CoordFreq {
    uint32_t idx;
    float shift;
};
struct CoordTaylor {
    uint32_t i_tail;
    float shift_tail;
    uint32_t i_head;
    float shift_head;
};

// Row stride (floats) of a staged profile: room for E and V (3-D) or the
// profile (2-D), and for the circular extension of the prefix sum; odd.
__host__ __device__ inline uint32_t row_stride(uint32_t nbins, bool is3d, uint32_t wmax) {
    uint32_t need = is3d ? 2 * nbins : nbins;
    if (nbins + wmax > need) {
        need = nbins + wmax;
    }
    return need | 1u;
}

// Scores the profile staged at r (stride-padded row) in place.
__device__ __forceinline__ void score_row(float* r, uint32_t nbins, bool is3d,
                                          float inv_stdnoise, const ScoreParams& sp, int mode,
                                          float* out) {
    float acc = 0.0f;
    for (uint32_t j = 0; j < nbins; ++j) {
        float x = r[j];
        if (is3d) {
            const float inv_sqrt_v = __fdiv_rn(1.0f, __fsqrt_rn(r[nbins + j]));
            x = __fmul_rn(x, inv_sqrt_v);
        }
        acc = (j == 0) ? x : __fadd_rn(acc, x);
        r[j] = acc;
    }
    const float sum = acc;
    for (uint32_t k = 0; k < sp.wmax; ++k) {
        r[nbins + k] = __fadd_rn(r[k], sum);
    }
    float dm[LK_MAX_WIDTHS];
#pragma unroll
    for (int iw = 0; iw < LK_MAX_WIDTHS; ++iw) {
        dm[iw] = -FLT_MAX;
    }
    for (uint32_t i = 0; i < nbins; ++i) {
        const float ri = r[i];
#pragma unroll
        for (int iw = 0; iw < LK_MAX_WIDTHS; ++iw) {
            if (iw < static_cast<int>(sp.nwidths)) {
                const float d = __fsub_rn(r[i + sp.widths[iw]], ri);
                dm[iw] = (dm[iw] < d) ? d : dm[iw];
            }
        }
    }
    float best = -FLT_MAX;
#pragma unroll
    for (int iw = 0; iw < LK_MAX_WIDTHS; ++iw) {
        if (iw < static_cast<int>(sp.nwidths)) {
            const float base = __fsub_rn(__fmul_rn(sp.hb[iw], dm[iw]), __fmul_rn(sp.b[iw], sum));
            const float snr = __fmul_rn(base, inv_stdnoise);
            if (mode == LK_SCORE_PER_WIDTH) {
                out[iw] = snr;
            } else {
                best = (best < snr) ? snr : best;
            }
        }
    }
    if (mode == LK_SCORE_MAX) {
        out[0] = best;
    }
}

__global__ void score_kernel(const float* __restrict__ folds, uint64_t nprof, uint32_t nbins,
                             bool is3d, float inv_stdnoise, uint32_t rs, ScoreParams sp, int mode,
                             float* __restrict__ scores) {
    extern __shared__ float rows[];
    const uint32_t T = blockDim.x;
    const uint64_t p0 = static_cast<uint64_t>(blockIdx.x) * T;
    const uint32_t plen = is3d ? 2 * nbins : nbins;
    const uint64_t nhere = (nprof - p0) < T ? (nprof - p0) : T;
    const uint64_t nelem = nhere * plen;
    const float* src = folds + p0 * plen;
    for (uint64_t e = threadIdx.x; e < nelem; e += T) {
        const uint64_t p = e / plen;
        const uint32_t j = static_cast<uint32_t>(e - p * plen);
        rows[p * rs + j] = __ldg(src + e);
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const uint64_t p = p0 + threadIdx.x;
        const uint32_t nout = mode == LK_SCORE_PER_WIDTH ? sp.nwidths : 1;
        score_row(rows + static_cast<size_t>(threadIdx.x) * rs, nbins, is3d, inv_stdnoise, sp,
                  mode, scores + p * nout);
    }
}

// Final FFA level (one segment) merged straight into shared memory and
// scored; the final fold never reaches global memory.
template <bool TAYLOR>
__global__ void merge_score_kernel(const float* __restrict__ in, const void* __restrict__ coords,
                                   uint64_t ncur, uint64_t nprev, uint32_t nbins, uint32_t rs,
                                   ScoreParams sp, int mode, float* __restrict__ scores) {
    extern __shared__ float rows[];
    const uint32_t T = blockDim.x;
    uint32_t* c_it = reinterpret_cast<uint32_t*>(rows + static_cast<size_t>(T) * rs);
    uint32_t* c_ih = c_it + T;
    uint32_t* c_st = c_ih + T;
    uint32_t* c_sh = c_st + T;
    const uint64_t p0 = static_cast<uint64_t>(blockIdx.x) * T;
    const uint32_t nhere = static_cast<uint32_t>((ncur - p0) < T ? (ncur - p0) : T);
    if (threadIdx.x < nhere) {
        const uint64_t c = p0 + threadIdx.x;
        if constexpr (TAYLOR) {
            const CoordTaylor k = reinterpret_cast<const CoordTaylor*>(coords)[c];
            c_it[threadIdx.x] = k.i_tail;
            c_ih[threadIdx.x] = k.i_head;
            c_st[threadIdx.x] = dev::shift_bins(k.shift_tail, nbins);
            c_sh[threadIdx.x] = dev::shift_bins(k.shift_head, nbins);
        } else {
            const CoordFreq k = reinterpret_cast<const CoordFreq*>(coords)[c];
            c_it[threadIdx.x] = k.idx;
            c_ih[threadIdx.x] = k.idx;
            c_st[threadIdx.x] = 0;
            c_sh[threadIdx.x] = dev::shift_bins(k.shift, nbins);
        }
    }
    __syncthreads();
    const uint32_t plen = 2 * nbins;
    const float* head_base = in + nprev * plen;  // segment 1 of the previous level
    // All threads sweep the block's rows; consecutive threads cover
    // consecutive output bins of one row (coalesced, rotated reads).
    const uint64_t nelem = static_cast<uint64_t>(nhere) * plen;
#pragma unroll 4
    for (uint64_t e = threadIdx.x; e < nelem; e += T) {
        const uint32_t p = static_cast<uint32_t>(e / plen);
        const uint32_t el = static_cast<uint32_t>(e - static_cast<uint64_t>(p) * plen);
        const uint32_t r = el >= nbins ? nbins : 0;
        const uint32_t j = el - r;
        const uint32_t st = c_st[p], sh = c_sh[p];
        const uint32_t jt = j >= st ? j - st : j + nbins - st;
        const uint32_t jh = j >= sh ? j - sh : j + nbins - sh;
        const float t = __ldg(in + static_cast<uint64_t>(c_it[p]) * plen + r + jt);
        const float h = __ldg(head_base + static_cast<uint64_t>(c_ih[p]) * plen + r + jh);
        rows[static_cast<size_t>(p) * rs + el] = __fadd_rn(t, h);
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const uint64_t p = p0 + threadIdx.x;
        const uint32_t nout = mode == LK_SCORE_PER_WIDTH ? sp.nwidths : 1;
        score_row(rows + static_cast<size_t>(threadIdx.x) * rs, nbins, true, 1.0f, sp, mode,
                  scores + p * nout);
    }
}

// Profiles per block so that the staged rows fit comfortably in shared memory.
uint32_t profiles_per_block(uint32_t rs, size_t extra_per_profile) {
    const size_t per = static_cast<size_t>(rs) * sizeof(float) + extra_per_profile;
    uint32_t T = 128;
    while (T > 32 && T * per > 100 * 1024) {
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

}  // namespace

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
    const uint32_t rs = row_stride(nbins, is3d, sp.wmax);
    const uint32_t T = profiles_per_block(rs, 0);
    const size_t smem = static_cast<size_t>(T) * rs * sizeof(float);
    set_smem(score_kernel, smem);
    const auto blocks = static_cast<unsigned>((nprof + T - 1) / T);
    score_kernel<<<blocks, T, smem, s>>>(d_folds, nprof, nbins, is3d, inv_stdnoise, rs, sp, mode,
                                         d_scores);
    LK_CUDA(cudaGetLastError());
}

void merge_score_level(const float* d_in, const void* d_coords, bool taylor,
                       uint64_t ncoords_cur, uint64_t ncoords_prev, uint32_t nbins,
                       const ScoreParams& sp, int mode, float* d_scores, cudaStream_t s) {
    if (ncoords_cur == 0) {
        return;
    }
    const uint32_t rs = row_stride(nbins, true, sp.wmax);
    const uint32_t T = profiles_per_block(rs, 4 * sizeof(uint32_t));
    const size_t smem = static_cast<size_t>(T) * (rs * sizeof(float) + 4 * sizeof(uint32_t));
    const auto blocks = static_cast<unsigned>((ncoords_cur + T - 1) / T);
    if (taylor) {
        set_smem(merge_score_kernel<true>, smem);
        merge_score_kernel<true><<<blocks, T, smem, s>>>(d_in, d_coords, ncoords_cur,
                                                         ncoords_prev, nbins, rs, sp, mode,
                                                         d_scores);
    } else {
        set_smem(merge_score_kernel<false>, smem);
        merge_score_kernel<false><<<blocks, T, smem, s>>>(d_in, d_coords, ncoords_cur,
                                                          ncoords_prev, nbins, rs, sp, mode,
                                                          d_scores);
    }
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
