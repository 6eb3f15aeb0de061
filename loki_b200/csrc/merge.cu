// One hierarchical merge level of the FFA:
//
//   out[s, c, r, j] = in[2s,   tail(c), r, (j - st(c)) mod nbins]
//                   + in[2s+1, head(c), r, (j - sh(c)) mod nbins]
//
// for r in {E, V}. Freq-only plans (FFACoordFreq) use tail = head = idx and an
// unshifted tail (lib/kernels.cpp:118-146, 722-827); Taylor plans (FFACoord)
// shift both halves (lib/kernels.cpp:71-112, 829-940). Each output element is
// one FP32 add of the same two operands as the reference, so results are
// bit-identical.
//
// Work split: a block covers up to kCoordsPerBlock consecutive frequency cells
// of one "outer" row (the higher-derivative cells: accel, or jerk x accel) of
// one segment; a warp handles one output row pair at a time with lanes
// striding over the 2*nbins elements (each warp instruction reads one rotated,
// contiguous 128-byte span). Blocks are numbered frequency-tile-major, so the
// outer rows that read the same parent rows run at the same time and share
// them through L2.
#include <algorithm>
#include <type_traits>

#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_merge.cuh"

namespace lk {

namespace {

constexpr int kWarp = 32;
constexpr int kThreads = 256;
constexpr uint32_t kCoordsPerBlock = 64;

// TIn / TOut: float or __nv_bfloat16 storage; every add is FP32.
template <bool TAYLOR, class TIn, class TOut>
__global__ void __launch_bounds__(kThreads)
    merge_kernel(const TIn* __restrict__ in, TOut* __restrict__ out,
                 const void* __restrict__ coords, uint32_t n_inner, uint32_t n_outer,
                 uint64_t nprev, uint32_t nbins) {
    const uint32_t tiles = (n_inner + kCoordsPerBlock - 1) / kCoordsPerBlock;
    const uint32_t tile = blockIdx.x / n_outer;
    const uint32_t outer = blockIdx.x - tile * n_outer;
    const uint64_t s = blockIdx.y;
    const uint64_t ncur = static_cast<uint64_t>(n_inner) * n_outer;
    const uint32_t row = 2 * nbins;
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    (void)tiles;
    const uint32_t j0 = tile * kCoordsPerBlock;
    const uint32_t j1 = min(j0 + kCoordsPerBlock, n_inner);
    for (uint32_t jf = j0 + warp; jf < j1; jf += kThreads / kWarp) {
        const uint64_t c = static_cast<uint64_t>(outer) * n_inner + jf;
        const MergeCoord mc = load_merge_coord<TAYLOR>(coords, c, nbins);
        const TIn* tail = in + ((2 * s) * nprev + mc.it) * row;
        const TIn* head = in + ((2 * s + 1) * nprev + mc.ih) * row;
        TOut* o = out + (s * ncur + c) * row;
        for (uint32_t e = lane; e < row; e += kWarp) {
            const uint32_t r = e >= nbins ? nbins : 0;
            const uint32_t j = e - r;
            const uint32_t jt = j >= mc.st ? j - mc.st : j + nbins - mc.st;
            const uint32_t jh = j >= mc.sh ? j - mc.sh : j + nbins - mc.sh;
            o[e] = dev::Store<TOut>::from_float(
                __fadd_rn(dev::Store<TIn>::load(tail + r + jt), dev::Store<TIn>::load(head + r + jh)));
        }
    }
}

// Loads-in-flight form for nbins <= 32 * NJ (NJ = 1, 2, 4): a warp takes PB
// output rows at a time, loads their coordinates with one lane each, issues
// every tail and head load of the PB rows (NJ bins per lane and row), then
// adds and stores. The first form keeps two loads in flight per lane and is
// latency-bound; this one keeps 4 * PB * NJ.
template <bool TAYLOR, class TIn, class TOut, int NJ, int PB>
__global__ void __launch_bounds__(kThreads)
    merge_kernel_mlp(const TIn* __restrict__ in, TOut* __restrict__ out,
                     const void* __restrict__ coords, uint32_t n_inner, uint32_t n_outer,
                     uint64_t nprev, uint32_t nbins) {
    const uint32_t tile = blockIdx.x / n_outer;
    const uint32_t outer = blockIdx.x - tile * n_outer;
    const uint64_t s = blockIdx.y;
    const uint64_t ncur = static_cast<uint64_t>(n_inner) * n_outer;
    const uint32_t row = 2 * nbins;
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const uint32_t j0 = tile * kCoordsPerBlock;
    const uint32_t j1 = min(j0 + kCoordsPerBlock, n_inner);
    const TIn* tail_base = in + (2 * s) * nprev * row;
    const TIn* head_base = in + (2 * s + 1) * nprev * row;
    TOut* out_base = out + (s * ncur + static_cast<uint64_t>(outer) * n_inner) * row;
    for (uint32_t p0 = j0 + warp * PB; p0 < j1; p0 += (kThreads / kWarp) * PB) {
        MergeCoord mine{0, 0, 0, 0};
        if (lane < PB && p0 + lane < j1) {
            mine = load_merge_coord<TAYLOR>(coords, static_cast<uint64_t>(outer) * n_inner + p0 + lane,
                                            nbins);
        }
        float te[PB][NJ], tv[PB][NJ], he[PB][NJ], hv[PB][NJ];
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            const uint32_t it = __shfl_sync(0xffffffffu, mine.it, q);
            const uint32_t ih = __shfl_sync(0xffffffffu, mine.ih, q);
            const uint32_t st = __shfl_sync(0xffffffffu, mine.st, q);
            const uint32_t sh = __shfl_sync(0xffffffffu, mine.sh, q);
            const bool live = p0 + q < j1;
            const TIn* tail = tail_base + static_cast<uint64_t>(it) * row;
            const TIn* head = head_base + static_cast<uint64_t>(ih) * row;
#pragma unroll
            for (int u = 0; u < NJ; ++u) {
                const uint32_t jr = lane + 32u * u;
                const bool ok = live && jr < nbins;
                const uint32_t j = ok ? jr : 0u;  // keep every address inside the rows
                const uint32_t jt = j >= st ? j - st : j + nbins - st;
                const uint32_t jh = j >= sh ? j - sh : j + nbins - sh;
                te[q][u] = ok ? dev::Store<TIn>::load(tail + jt) : 0.0f;
                tv[q][u] = ok ? dev::Store<TIn>::load(tail + nbins + jt) : 0.0f;
                he[q][u] = ok ? dev::Store<TIn>::load(head + jh) : 0.0f;
                hv[q][u] = ok ? dev::Store<TIn>::load(head + nbins + jh) : 0.0f;
            }
        }
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            if (p0 + q < j1) {
                TOut* o = out_base + static_cast<uint64_t>(p0 + q) * row;
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    const uint32_t j = lane + 32u * u;
                    if (j < nbins) {
                        o[j] = dev::Store<TOut>::from_float(__fadd_rn(te[q][u], he[q][u]));
                        o[nbins + j] = dev::Store<TOut>::from_float(__fadd_rn(tv[q][u], hv[q][u]));
                    }
                }
            }
        }
    }
}

// nbins = NB in {32, 64, 128}: rotations are (j - shift) & (NB - 1), every
// lane's bins are in range, E and V of a row share one address register
// (V at an immediate offset), and stores use immediate offsets from one
// per-row base, which halves the integer work per element of
// merge_kernel_mlp (that kernel is issue-bound on its index arithmetic).
template <bool TAYLOR, class TIn, class TOut, int NB, int PB>
__global__ void __launch_bounds__(kThreads)
    merge_kernel_p2(const TIn* __restrict__ in, TOut* __restrict__ out,
                    const void* __restrict__ coords, uint32_t n_inner, uint32_t n_outer,
                    uint64_t nprev) {
    constexpr int NJ = NB / 32;
    constexpr uint32_t row = 2 * NB;
    const uint32_t tile = blockIdx.x / n_outer;
    const uint32_t outer = blockIdx.x - tile * n_outer;
    const uint64_t s = blockIdx.y;
    const uint64_t ncur = static_cast<uint64_t>(n_inner) * n_outer;
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const uint32_t j0 = tile * kCoordsPerBlock;
    const uint32_t j1 = min(j0 + kCoordsPerBlock, n_inner);
    const TIn* tail_base = in + (2 * s) * nprev * row;
    const TIn* head_base = in + (2 * s + 1) * nprev * row;
    TOut* out_base = out + (s * ncur + static_cast<uint64_t>(outer) * n_inner) * row + lane;
    for (uint32_t p0 = j0 + warp * PB; p0 < j1; p0 += (kThreads / kWarp) * PB) {
        MergeCoord mine{0, 0, 0, 0};
        if (lane < PB && p0 + lane < j1) {
            mine = load_merge_coord<TAYLOR>(coords, static_cast<uint64_t>(outer) * n_inner + p0 + lane,
                                            NB);
        }
        float te[PB][NJ], tv[PB][NJ], he[PB][NJ], hv[PB][NJ];
#pragma unroll
        for (int q = 0; q < PB; ++q) {
            const uint32_t it = __shfl_sync(0xffffffffu, mine.it, q);
            const uint32_t ih = __shfl_sync(0xffffffffu, mine.ih, q);
            const uint32_t st = __shfl_sync(0xffffffffu, mine.st, q);
            const uint32_t sh = __shfl_sync(0xffffffffu, mine.sh, q);
            // rows of a coordinate past j1 read row 0 (in range) and are not stored
            const bool live = p0 + q < j1;
            const TIn* tail = tail_base + static_cast<uint64_t>(live ? it : 0u) * row;
            const TIn* head = head_base + static_cast<uint64_t>(live ? ih : 0u) * row;
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
            if (p0 + q < j1) {
                TOut* o = out_base + static_cast<uint64_t>(p0 + q) * row;
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    o[32 * u] = dev::Store<TOut>::from_float(__fadd_rn(te[q][u], he[q][u]));
                    o[NB + 32 * u] = dev::Store<TOut>::from_float(__fadd_rn(tv[q][u], hv[q][u]));
                }
            }
        }
    }
}

}  // namespace

void merge_level(const void* d_in, void* d_out, const void* d_coords, bool taylor,
                 uint64_t n_inner, uint64_t n_outer, uint64_t ncoords_prev, uint64_t nsegments,
                 uint32_t nbins, cudaStream_t s, bool in_bf16, bool out_bf16, int pb) {
    require(n_inner > 0 && n_outer > 0, "empty merge level");
    const uint64_t tiles = (n_inner + kCoordsPerBlock - 1) / kCoordsPerBlock;
    require(tiles * n_outer <= 0x7fffffffULL && n_inner <= 0xffffffffULL &&
                n_outer <= 0xffffffffULL,
            "merge level too large for the launch grid");
    // Output segments on grid.y, at most 65535 per launch (batched series can
    // have more).
    const uint64_t row = 2ull * nbins;
    const uint64_t ncur = n_inner * n_outer;
    for (uint64_t s0 = 0; s0 < nsegments; s0 += 65535) {
        const uint64_t ns = std::min<uint64_t>(65535, nsegments - s0);
        dim3 grid(static_cast<unsigned>(tiles * n_outer), static_cast<unsigned>(ns));
        const uint64_t in_off = s0 * 2 * ncoords_prev * row;
        const uint64_t out_off = s0 * ncur * row;
        auto launch = [&](auto tin, auto tout) {
            using TIn = decltype(tin);
            using TOut = decltype(tout);
            const TIn* in = static_cast<const TIn*>(d_in) + in_off;
            TOut* out = static_cast<TOut*>(d_out) + out_off;
            const auto ni = static_cast<uint32_t>(n_inner);
            const auto no = static_cast<uint32_t>(n_outer);
            auto go = [&](auto kern) {
                kern<<<grid, kThreads, 0, s>>>(in, out, d_coords, ni, no, ncoords_prev, nbins);
            };
            auto go_p2 = [&](auto kern) {
                kern<<<grid, kThreads, 0, s>>>(in, out, d_coords, ni, no, ncoords_prev);
            };
            auto pick = [&](auto tg) {
                constexpr bool TG = decltype(tg)::value;
                // pb: output rows per warp in flight (0: 8 / 4 / 2 for nbins
                // 32 / 64 / 128, i.e. 16 loads of each kind per lane)
                if (nbins == 32) {
                    pb == 4    ? go_p2(merge_kernel_p2<TG, TIn, TOut, 32, 4>)
                    : pb == 16 ? go_p2(merge_kernel_p2<TG, TIn, TOut, 32, 16>)
                               : go_p2(merge_kernel_p2<TG, TIn, TOut, 32, 8>);
                } else if (nbins == 64) {
                    pb == 2   ? go_p2(merge_kernel_p2<TG, TIn, TOut, 64, 2>)
                    : pb == 8 ? go_p2(merge_kernel_p2<TG, TIn, TOut, 64, 8>)
                              : go_p2(merge_kernel_p2<TG, TIn, TOut, 64, 4>);
                } else if (nbins == 128) {
                    pb == 1   ? go_p2(merge_kernel_p2<TG, TIn, TOut, 128, 1>)
                    : pb == 4 ? go_p2(merge_kernel_p2<TG, TIn, TOut, 128, 4>)
                              : go_p2(merge_kernel_p2<TG, TIn, TOut, 128, 2>);
                } else if (nbins == 256) {
                    // the octave sweep's wider regions: one row per warp in
                    // flight (32 / 64 / 128 loads per lane)
                    go_p2(merge_kernel_p2<TG, TIn, TOut, 256, 1>);
                } else if (nbins == 512) {
                    go_p2(merge_kernel_p2<TG, TIn, TOut, 512, 1>);
                } else if (nbins == 1024) {
                    go_p2(merge_kernel_p2<TG, TIn, TOut, 1024, 1>);
                } else if (nbins <= 32) {
                    go(merge_kernel_mlp<TG, TIn, TOut, 1, 8>);
                } else if (nbins <= 64) {
                    go(merge_kernel_mlp<TG, TIn, TOut, 2, 4>);
                } else if (nbins <= 128) {
                    go(merge_kernel_mlp<TG, TIn, TOut, 4, 2>);
                } else {
                    go(merge_kernel<TG, TIn, TOut>);
                }
            };
            if (taylor) {
                pick(std::true_type{});
            } else {
                pick(std::false_type{});
            }
        };
        if (!in_bf16 && !out_bf16) {
            launch(float{}, float{});
        } else if (!in_bf16) {
            launch(float{}, __nv_bfloat16{});
        } else if (out_bf16) {
            launch(__nv_bfloat16{}, __nv_bfloat16{});
        } else {
            launch(__nv_bfloat16{}, float{});
        }
        LK_CUDA(cudaGetLastError());
    }
}

}  // namespace lk
