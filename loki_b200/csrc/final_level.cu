// Final FFA level fused with boxcar scoring, for 32, 64 or 128 bins and
// strictly increasing widths of at most 32 bins (the reference's default
// width trials and the benchmark widths), with the search's candidate counts
// fused in.
//
// Same arithmetic as merge_score_kernel (score.cu), which stays the path for
// every other case (reference: snr_boxcar_impl, lib/score.cpp:95-172;
// circular_prefix_sum / diff_max, lib/utils.cpp:22-67):
//   x_j    = E_j * (1 / sqrt(V_j))           E, V = tail + head rows (FP32 adds)
//   p      = sequential inclusive prefix sum of x, extended by wmax bins
//   dmax_w = max_i (p[i + w] - p[i])
//   snr_w  = (h_w + b_w) * dmax_w - b_w * p[nbins - 1]
// What differs is how the work is laid out:
//  * 1 / sqrt(V) comes from a table for V an exact integer below 2^19 (a
//    variance series of ones makes every V a sample count): the table entry
//    is the same correctly rounded rcp(sqrt(n)) the direct path computes, so
//    the product is the same; other V take the direct path;
//  * each thread scores one cell from its staged prefix row: the row is read
//    into registers 16 positions (plus the widest width) at a time and every
//    width w up to the bucket WM (8, 16 or 32) is a compile-time register
//    offset, taken when bit w of the width mask is set; window differences
//    are the same IEEE subtracts, reduced by a tree of three-input maxima
//    (max.f32 a, b, c), which return the same value as the reference's
//    `(m < d) ? d : m` scan (NaN differences are skipped by both) except
//    possibly for the sign of a zero maximum, so a zero maximum is
//    recomputed with the reference's rule; rows are read and the prefix
//    sums written two bins per 64-bit shared-memory access;
//  * with a count target, each block counts its scores >= thr; a block's
//    cells are contiguous in flat score order, so the candidate list is an
//    exclusive scan of the block counts plus an ordered scatter of the blocks
//    that have candidates (compact_ranges), without a separate counting pass.
#include <cfloat>
#include <cmath>

#include "lk_block.cuh"
#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_merge.cuh"
#include "lk_score.cuh"

namespace lk {

namespace {

constexpr int kWarp = 32;
constexpr int kMaxW = 32;  // largest width of the masked path

__global__ void norm_table_kernel(float* __restrict__ tab, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        tab[i] = __frcp_rn(__fsqrt_rn(__uint2float_rn(i)));
    }
}

// max of three (sm_100 three-input max.f32: the largest non-NaN input, as
// two nested fmaxf).
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Exact reference maximum (first maximum kept) of p[i + w] - p[i].
__device__ __noinline__ float dmax_exact(const float* r, uint32_t w, uint32_t nbins) {
    float m = -FLT_MAX;
    for (uint32_t i = 0; i < nbins; ++i) {
        const float d = __fsub_rn(r[i + w], r[i]);
        m = (m < d) ? d : m;
    }
    return m;
}

using sc::kFixedMask16;

// WM: largest width the kernel handles (8, 16 or 32; the width mask has no
// bit above it), so only WM width bodies are generated. CH: window chunk.
// TAB: 1 / sqrt(V) from the table where V is an exact integer inside it.
// FM: the width mask as a compile-time constant (mp.wmask == FM), or 0 to
// test mp.wmask at run time.
template <bool TAYLOR, int NB, int PB, class TIn, int WM, bool TAB, uint64_t FM>
__global__ void __launch_bounds__(128, 5)
    merge_score_wm_kernel(const TIn* __restrict__ in, const void* __restrict__ coords,
                          uint32_t n_inner, uint32_t n_outer, uint64_t nprev, MaskScoreParams mp,
                          int mode, float* __restrict__ scores, float* __restrict__ cmax,
                          const float* __restrict__ tab, float thr, uint32_t* __restrict__ counts) {
    constexpr int NJ = NB / kWarp;      // bins per lane in phase 1
    // Row stride, room for every window read: NB + WM + 2 floats, so that
    // rows start on 8 bytes and half the stride is odd -- the 64-bit loads
    // of 16 threads (one row each) then fall on distinct bank pairs.
    constexpr int RS = NB + WM + 2;
    constexpr int CH = 16;
    static_assert(NB % CH == 0 && WM <= kMaxW, "chunking");
    extern __shared__ float rows[];
    const uint32_t nout = mode == LK_SCORE_PER_WIDTH ? mp.nwidths : 1;
    in += static_cast<uint64_t>(blockIdx.y) * 2 * nprev * 2 * NB;
    scores += static_cast<uint64_t>(blockIdx.y) * n_inner * n_outer * nout;
    if (cmax != nullptr) {
        cmax += static_cast<uint64_t>(blockIdx.y) * n_inner * n_outer;
    }
    const uint32_t T = blockDim.x;
    const uint32_t tiles = (n_inner + T - 1) / T;
    const uint32_t tile = blockIdx.x / n_outer;
    const uint32_t outer = blockIdx.x - tile * n_outer;
    const uint32_t j0 = tile * T;
    const uint32_t nhere = min(T, n_inner - j0);
    const uint64_t c0 = static_cast<uint64_t>(outer) * n_inner + j0;
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    constexpr uint32_t plen = 2 * NB;
    const TIn* head_base = in + nprev * plen;

    // Phase 1: a warp takes PB cells at a time, every load in flight, lanes
    // over bins; normalised profiles into shared memory.
    for (uint32_t p0 = warp * PB; p0 < nhere; p0 += (T / kWarp) * PB) {
        MergeCoord mine{0, 0, 0, 0};
        if (lane < PB && p0 + lane < nhere) {
            mine = load_merge_coord<TAYLOR>(coords, c0 + p0 + lane, NB);
        }
        float se[PB][NJ], sv[PB][NJ];
        {
            float te[PB][NJ], tv[PB][NJ], he[PB][NJ], hv[PB][NJ];
#pragma unroll
            for (int q = 0; q < PB; ++q) {
                const uint32_t it = __shfl_sync(0xffffffffu, mine.it, q);
                const uint32_t ih = __shfl_sync(0xffffffffu, mine.ih, q);
                const uint32_t st = __shfl_sync(0xffffffffu, mine.st, q);
                const uint32_t sh = __shfl_sync(0xffffffffu, mine.sh, q);
                const bool live = p0 + q < nhere;
                // rows past nhere read row 0 (in range) and are not used
                const TIn* tail = live ? in + static_cast<uint64_t>(it) * plen : in;
                const TIn* head = live ? head_base + static_cast<uint64_t>(ih) * plen : head_base;
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    const uint32_t j = lane + 32u * u;
                    const TIn* pt = tail + ((j - st) & (NB - 1));
                    const TIn* ph = head + ((j - sh) & (NB - 1));
                    te[q][u] = dev::Store<TIn>::load(pt);
                    tv[q][u] = dev::Store<TIn>::load(pt + NB);
                    he[q][u] = dev::Store<TIn>::load(ph);
                    hv[q][u] = dev::Store<TIn>::load(ph + NB);
                }
            }
#pragma unroll
            for (int q = 0; q < PB; ++q) {
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    se[q][u] = __fadd_rn(te[q][u], he[q][u]);
                    sv[q][u] = __fadd_rn(tv[q][u], hv[q][u]);
                }
            }
        }
        if constexpr (TAB) {
            // every table read in flight before the first product
            float inv[PB][NJ];
            bool ok[PB][NJ];
#pragma unroll
            for (int q = 0; q < PB; ++q) {
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    const uint32_t n = __float2uint_rz(sv[q][u]);
                    ok[q][u] = n < kNormTableSize &&
                               __float_as_uint(__uint2float_rn(n)) == __float_as_uint(sv[q][u]);
                    inv[q][u] = __ldg(tab + (ok[q][u] ? n : 0u));
                }
            }
#pragma unroll
            for (int q = 0; q < PB; ++q) {
                if (p0 + q < nhere) {
                    float* dst = rows + static_cast<size_t>(p0 + q) * RS;
#pragma unroll
                    for (int u = 0; u < NJ; ++u) {
                        float x;
                        if (ok[q][u]) {
                            x = __fmul_rn(se[q][u], inv[q][u]);
                        } else {
                            x = sc::normalise(se[q][u], sv[q][u]);
                        }
                        dst[lane + 32u * u] = x;
                    }
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < PB; ++q) {
                if (p0 + q < nhere) {
                    float* dst = rows + static_cast<size_t>(p0 + q) * RS;
#pragma unroll
                    for (int u = 0; u < NJ; ++u) {
                        dst[lane + 32u * u] = sc::normalise(se[q][u], sv[q][u]);
                    }
                }
            }
        }
    }
    __syncthreads();

    // Phase 2: one thread per cell.
    uint32_t passed = 0;
    if (threadIdx.x < nhere) {
        float* r = rows + static_cast<size_t>(threadIdx.x) * RS;
        float2* r2 = reinterpret_cast<float2*>(r);
        // sequential inclusive prefix sum, two bins per 64-bit access
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
            // positions c .. c + CH + WM - 1 (inside the row); those past
            // NB + wmax - 1 are only used by widths above wmax (not taken)
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
                    // the chunk's 16 differences and the running maximum
                    // in a tree of three-input maxima (depth 3)
                    float d[CH];
#pragma unroll
                    for (int k = 0; k < CH; ++k) {
                        d[k] = __fsub_rn(win[k + w], win[k]);
                    }
                    static_assert(CH == 16, "tree below is for 16 differences");
                    const float m0 = fmax3(d[0], d[1], d[2]);
                    const float m1 = fmax3(d[3], d[4], d[5]);
                    const float m2 = fmax3(d[6], d[7], d[8]);
                    const float m3 = fmax3(d[9], d[10], d[11]);
                    const float m4 = fmax3(d[12], d[13], d[14]);
                    const float n0 = fmax3(m0, m1, m2);
                    const float n1 = fmax3(m3, m4, d[15]);
                    dm[w] = fmax3(dm[w], n0, n1);
                }
            }
        }
        const uint64_t c = c0 + threadIdx.x;
        float best = -FLT_MAX;
#pragma unroll
        for (int w = 1; w <= WM; ++w) {
            if (taken(w)) {
                float d = dm[w];
                if (d == 0.0f) {
                    d = dmax_exact(r, static_cast<uint32_t>(w), NB);
                }
                // ((h + b) dmax - b sum) times 1 / stdnoise = 1 (3-D folds)
                const float snr = __fsub_rn(__fmul_rn(mp.hb[w], d), __fmul_rn(mp.b[w], sum));
                if (mode == LK_SCORE_PER_WIDTH) {
                    scores[c * nout + mp.slot[w]] = snr;
                }
                passed += snr >= thr ? 1u : 0u;
                best = (best < snr) ? snr : best;
            }
        }
        if (mode == LK_SCORE_MAX) {
            scores[c] = best;
        }
        if (cmax != nullptr) {
            cmax[c] = best;
        }
    }
    if (counts != nullptr) {
        __shared__ uint32_t ws[32];
        uint32_t total;
        blk::block_exclusive_scan(passed, ws, &total);
        if (threadIdx.x == 0) {
            counts[(static_cast<uint64_t>(blockIdx.y) * n_outer + outer) * tiles + tile] = total;
        }
    }
}

// Ordered scatter of the scores >= thr of one range (a final-level block's
// cells, flat order), at the range's offset from the exclusive scan.
__global__ void range_scatter_kernel(const float* __restrict__ x, const uint32_t* __restrict__ counts,
                                     const uint64_t* __restrict__ offsets, uint32_t n_inner,
                                     uint32_t n_outer, uint32_t tiles, uint32_t T, uint32_t nw,
                                     float thr, uint32_t* __restrict__ idx, float* __restrict__ vals,
                                     uint64_t max_out) {
    if (counts[blockIdx.x] == 0) {
        return;  // uniform per block
    }
    __shared__ uint32_t ws[32];
    const uint32_t k = blockIdx.x;
    const uint32_t tile = k % tiles;
    const uint64_t series_outer = k / tiles;  // series * n_outer + outer
    const uint64_t ncells_series = static_cast<uint64_t>(n_inner) * n_outer;
    const uint64_t series = series_outer / n_outer;
    const uint64_t outer = series_outer - series * n_outer;
    const uint32_t j0 = tile * T;
    const uint32_t nhere = min(T, n_inner - j0);
    const uint64_t base = (series * ncells_series + outer * n_inner + j0) * nw;
    const uint32_t len = nhere * nw;
    uint64_t pos = offsets[k];
    for (uint32_t s0 = 0; s0 < len; s0 += blockDim.x * 4) {
        float v[4];
        uint32_t c = 0;
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            const uint32_t i = s0 + threadIdx.x * 4 + q;
            v[q] = i < len ? x[base + i] : 0.0f;
            c += (i < len && v[q] >= thr) ? 1u : 0u;
        }
        uint32_t total;
        uint64_t p = pos + blk::block_exclusive_scan(c, ws, &total);
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            const uint32_t i = s0 + threadIdx.x * 4 + q;
            if (i < len && v[q] >= thr) {
                if (p < max_out) {
                    idx[p] = static_cast<uint32_t>(base + i);
                    vals[p] = v[q];
                }
                ++p;
            }
        }
        pos += total;
        __syncthreads();  // ws reused by the next chunk's scan
    }
}

}  // namespace

void norm_table_fill(float* d_tab, cudaStream_t s) {
    norm_table_kernel<<<(kNormTableSize + 255) / 256, 256, 0, s>>>(d_tab, kNormTableSize);
    LK_CUDA(cudaGetLastError());
}

bool make_mask_score_params(const ScoreParams& sp, uint32_t nbins, MaskScoreParams* mp) {
    if (nbins != 32 && nbins != 64 && nbins != 128) {
        return false;
    }
    MaskScoreParams m{};
    uint32_t prev = 0;
    for (uint32_t i = 0; i < sp.nwidths; ++i) {
        const uint32_t w = sp.widths[i];
        if (w <= prev || w > static_cast<uint32_t>(kMaxW)) {
            return false;  // not strictly increasing, or wider than the masked path
        }
        prev = w;
        m.wmask |= 1ull << w;
        m.hb[w] = sp.hb[i];
        m.b[w] = sp.b[i];
        m.slot[w] = static_cast<uint8_t>(i);
    }
    m.nwidths = sp.nwidths;
    m.wmax = sp.wmax;
    *mp = m;
    return true;
}

uint32_t final_level_cells_per_block() { return 128; }

void merge_score_level_wm(const void* d_in, const void* d_coords, bool taylor, uint64_t n_inner,
                          uint64_t n_outer, uint64_t ncoords_prev, uint32_t nbins,
                          const MaskScoreParams& mp, int mode, float* d_scores, cudaStream_t s,
                          uint64_t nbatch, bool in_bf16, float* d_cmax, const float* d_tab,
                          float count_thr, uint32_t* d_counts, bool use_table) {
    require(nbatch >= 1 && nbatch <= 65535, "nbatch must lie in [1, 65535]");
    if (n_inner == 0 || n_outer == 0) {
        return;
    }
    const uint32_t T = final_level_cells_per_block();
    const uint64_t tiles = (n_inner + T - 1) / T;
    require(tiles * n_outer <= 0x7fffffffULL && n_inner <= 0xffffffffULL,
            "final level too large for the launch grid");
    const auto blocks = static_cast<unsigned>(tiles * n_outer);
    require(d_tab != nullptr || !use_table, "internal: no normalisation table");
    const bool fixed16 = mp.wmask == kFixedMask16 && mp.wmax == 16;
    auto go2 = [&](auto tg, auto tin, auto nbc, auto wmc, auto tabc) {
        constexpr bool TG = decltype(tg)::value;
        using TI = decltype(tin);
        constexpr int NB = decltype(nbc)::value;
        constexpr int WM = decltype(wmc)::value;
        constexpr bool TB = decltype(tabc)::value;
        constexpr int PB = NB == 128 ? 4 : 8;
        auto kern = merge_score_wm_kernel<TG, NB, PB, TI, WM, TB, 0>;
        if constexpr (WM == 16) {
            if (fixed16) {
                kern = merge_score_wm_kernel<TG, NB, PB, TI, WM, TB, kFixedMask16>;
            }
        }
        const size_t smem = static_cast<size_t>(T) * (NB + WM + 2) * sizeof(float);
        sc::set_smem(kern, smem);
        kern<<<dim3(blocks, static_cast<unsigned>(nbatch)), T, smem, s>>>(
            static_cast<const TI*>(d_in), d_coords, static_cast<uint32_t>(n_inner),
            static_cast<uint32_t>(n_outer), ncoords_prev, mp, mode, d_scores, d_cmax, d_tab,
            count_thr, d_counts);
    };
    auto go = [&](auto tg, auto tin, auto nbc) {
        auto by_tab = [&](auto wmc) {
            use_table ? go2(tg, tin, nbc, wmc, std::true_type{}) : go2(tg, tin, nbc, wmc, std::false_type{});
        };
        if (mp.wmax <= 8) {
            by_tab(std::integral_constant<int, 8>{});
        } else if (mp.wmax <= 16) {
            by_tab(std::integral_constant<int, 16>{});
        } else {
            by_tab(std::integral_constant<int, 32>{});
        }
    };
    auto by_nb = [&](auto tg, auto tin) {
        if (nbins == 32) {
            go(tg, tin, std::integral_constant<int, 32>{});
        } else if (nbins == 64) {
            go(tg, tin, std::integral_constant<int, 64>{});
        } else {
            go(tg, tin, std::integral_constant<int, 128>{});
        }
    };
    if (taylor) {
        in_bf16 ? by_nb(std::true_type{}, __nv_bfloat16{}) : by_nb(std::true_type{}, float{});
    } else {
        in_bf16 ? by_nb(std::false_type{}, __nv_bfloat16{}) : by_nb(std::false_type{}, float{});
    }
    LK_CUDA(cudaGetLastError());
}

uint64_t final_level_blocks(uint64_t n_inner, uint64_t n_outer, uint64_t nbatch) {
    const uint64_t T = final_level_cells_per_block();
    return ((n_inner + T - 1) / T) * n_outer * nbatch;
}

void compact_ranges(const float* d_scores, const uint32_t* d_counts, uint64_t* d_offsets,
                    uint64_t n_inner, uint64_t n_outer, uint64_t nbatch, uint32_t nw, float thr,
                    uint32_t* d_idx, float* d_vals, uint64_t max_out, uint64_t* d_count,
                    cudaStream_t s) {
    const uint64_t nblocks = final_level_blocks(n_inner, n_outer, nbatch);
    require(nblocks <= 0x7fffffffULL, "too many compaction ranges");
    require(n_inner * n_outer * nbatch * nw <= 0xffffffffULL,
            "compaction indices are 32-bit: scores must number < 2^32");
    const uint32_t T = final_level_cells_per_block();
    const auto tiles = static_cast<uint32_t>((n_inner + T - 1) / T);
    scan_counts(d_counts, nblocks, d_offsets, d_count, s);
    range_scatter_kernel<<<static_cast<unsigned>(nblocks), 256, 0, s>>>(
        d_scores, d_counts, d_offsets, static_cast<uint32_t>(n_inner),
        static_cast<uint32_t>(n_outer), tiles, T, nw, thr, d_idx, d_vals, max_out);
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
