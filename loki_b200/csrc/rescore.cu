// Exact FP32 rescoring of selected final FFA cells.
//
// With BF16 storage of the intermediate levels, the final-level scores carry
// rounding error. A search keeps its candidate set identical to the all-FP32
// path by rescoring every cell whose approximate best S/N lies within a margin
// of the threshold: this kernel rebuilds the final fold of such a cell from
// the FP32 level-0 fold (which the BF16 path keeps) with the same FP32 adds,
// in the same tree, as the all-FP32 merge levels, then scores it with the same
// boxcar code. The result is bit-identical to the all-FP32 score of that cell.
//
// The merge tree of one final cell. merge level l computes
//   F_l[s, c, r, j] = F_{l-1}[2s, tail(c), r, (j - st(c)) mod n]
//                   + F_{l-1}[2s+1, head(c), r, (j - sh(c)) mod n]
// (lib/kernels.cpp:71-146 of the reference), so the final value at bin j is a
// perfect binary tree of adds over the 2^(L-1) level-0 segments, leaf s read
// at row leaf_idx[s] and bin (j - leaf_off[s]) mod n, where leaf_off is the
// sum of the shifts along the path. A block expands the path top-down once per
// cell (leaf table in shared memory), then each thread reduces one (row, bin)
// over a quarter of the leaves (an aligned subtree) bottom-up with a
// binary-counter stack, and the four subtree totals are added as the tree's
// top two levels. This groups the adds exactly as the level-by-level merges
// do (IEEE addition is commutative, so the operand order of each add does not
// matter; the grouping does).
#include <algorithm>

#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_merge.cuh"
#include "lk_score.cuh"

namespace lk {

namespace {

constexpr uint32_t kThreads = 512;
constexpr uint32_t kLane = 128;  // threads per leaf part
constexpr uint32_t kParts = kThreads / kLane;
constexpr uint32_t kGroup = 8;  // leaves loaded before their adds (ILP)

struct Leaf {
    uint32_t idx;
    uint32_t off;
};

template <bool TAYLOR, int NW, int NB>
__global__ void __launch_bounds__(kThreads)
    rescore_kernel(const float* __restrict__ fold0, RescoreTree t, ScoreParams sp, uint32_t rs,
                   const uint32_t* __restrict__ cells, const uint64_t* __restrict__ d_count,
                   uint64_t max_cells, float* __restrict__ scores) {
    extern __shared__ unsigned char smem_raw[];
    const uint32_t nbins = t.nbins;
    const uint32_t nleaves = 1u << (t.n_levels - 1);
    Leaf* la = reinterpret_cast<Leaf*>(smem_raw);
    Leaf* lb = la + nleaves;
    float* ev = reinterpret_cast<float*>(lb + nleaves);  // [kParts][2 * nbins]
    float* row = ev + kParts * 2 * nbins;                // [rs]
    // The leaves split into nparts aligned subtrees (parts of >= kGroup
    // leaves), each reduced by kLane threads; the part totals are then added
    // pairwise, which is the top of the same tree.
    const uint32_t nparts = nleaves >= kParts * kGroup ? kParts : 1;
    const uint32_t pleaves = nleaves / nparts;
    const uint32_t part = threadIdx.x / kLane;
    const uint64_t count = min(*d_count, max_cells);
    const uint32_t plen = 2 * nbins;
    for (uint64_t k = blockIdx.x; k < count; k += gridDim.x) {
        const uint64_t cell = cells[k];
        const uint64_t series = cell / t.ncoords_final;
        const uint64_t coord = cell - series * t.ncoords_final;
        // ---- top-down: leaf rows and composed shifts -------------------
        if (threadIdx.x == 0) {
            la[0] = Leaf{static_cast<uint32_t>(coord), 0u};
        }
        __syncthreads();
        Leaf* cur = la;
        Leaf* nxt = lb;
        for (uint32_t l = t.n_levels - 1, n = 1; l >= 1; --l, n *= 2) {
            for (uint32_t q = threadIdx.x; q < n; q += blockDim.x) {
                const Leaf p = cur[q];
                const MergeCoord mc = load_merge_coord<TAYLOR>(t.level_coords[l], p.idx, nbins);
                uint32_t ot = p.off + mc.st;
                uint32_t oh = p.off + mc.sh;
                ot = ot >= nbins ? ot - nbins : ot;
                oh = oh >= nbins ? oh - nbins : oh;
                nxt[2 * q] = Leaf{mc.it, ot};
                nxt[2 * q + 1] = Leaf{mc.ih, oh};
            }
            __syncthreads();
            Leaf* tmp = cur;
            cur = nxt;
            nxt = tmp;
        }
        // ---- bottom-up: FP32 add tree per (row, bin) ---------------------
        const float* base = fold0 + series * t.fold0_size;
        for (uint32_t e = threadIdx.x % kLane; part < nparts && e < plen; e += kLane) {
            const uint32_t r = e >= nbins ? nbins : 0;
            const uint32_t j = e - r;
            float stk[kRescoreMaxLevels];
            auto leaf_value = [&](uint32_t sl) {
                const uint32_t s = part * pleaves + sl;
                const Leaf lf = cur[s];
                const uint32_t jj = j >= lf.off ? j - lf.off : j + nbins - lf.off;
                return __ldg(base + (static_cast<uint64_t>(s) * t.ncoords0 + lf.idx) * plen + r +
                             jj);
            };
            float total;
            if (pleaves >= kGroup) {
                const uint32_t ngroups = pleaves / kGroup;
                for (uint32_t g = 0; g < ngroups; ++g) {
                    float v[kGroup];
#pragma unroll
                    for (uint32_t u = 0; u < kGroup; ++u) {
                        v[u] = leaf_value(g * kGroup + u);
                    }
                    // levels 1..3 of the tree inside the group
#pragma unroll
                    for (uint32_t w = 1; w < kGroup; w *= 2) {
#pragma unroll
                        for (uint32_t u = 0; u < kGroup; u += 2 * w) {
                            v[u] = __fadd_rn(v[u], v[u + w]);
                        }
                    }
                    float acc = v[0];
                    uint32_t b = 0;
                    while ((g >> b) & 1u) {
                        acc = __fadd_rn(stk[b], acc);
                        ++b;
                    }
                    stk[b] = acc;
                }
                total = stk[31 - __clz(ngroups)];
            } else {
                for (uint32_t q = 0; q < pleaves; ++q) {
                    float acc = leaf_value(q);
                    uint32_t b = 0;
                    while ((q >> b) & 1u) {
                        acc = __fadd_rn(stk[b], acc);
                        ++b;
                    }
                    stk[b] = acc;
                }
                total = stk[31 - __clz(pleaves)];
            }
            ev[part * plen + e] = total;
        }
        __syncthreads();
        for (uint32_t j = threadIdx.x; j < nbins; j += blockDim.x) {
            float fe, fv;
            if (nparts == kParts) {
                static_assert(kParts == 4, "part totals are added as a 4-leaf tree");
                fe = __fadd_rn(__fadd_rn(ev[j], ev[plen + j]),
                               __fadd_rn(ev[2 * plen + j], ev[3 * plen + j]));
                fv = __fadd_rn(__fadd_rn(ev[nbins + j], ev[plen + nbins + j]),
                               __fadd_rn(ev[2 * plen + nbins + j], ev[3 * plen + nbins + j]));
            } else {
                fe = ev[j];
                fv = ev[nbins + j];
            }
            row[j] = sc::normalise(fe, fv);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            sc::score_row_any<NB, NW>(row, nbins, 1.0f, sp, LK_SCORE_PER_WIDTH,
                                      scores + cell * sp.nwidths);
        }
        __syncthreads();
    }
}

}  // namespace

void rescore_cells(const float* d_fold0, const RescoreTree& t, bool taylor, const ScoreParams& sp,
                   const uint32_t* d_cells, const uint64_t* d_count, uint64_t max_cells,
                   float* d_scores, cudaStream_t s) {
    require(t.n_levels >= 2 && t.n_levels <= kRescoreMaxLevels, "rescore: level count out of range");
    require((1ull << (t.n_levels - 1)) <= kRescoreMaxLeaves, "rescore: too many level-0 segments");
    if (max_cells == 0) {
        return;
    }
    const uint32_t nleaves = 1u << (t.n_levels - 1);
    const uint32_t rs = sc::row_stride(t.nbins, sp.wmax);
    const size_t smem = 2 * nleaves * sizeof(Leaf) + (kParts * 2 * t.nbins + rs) * sizeof(float);
    require(smem <= 200 * 1024, "rescore: nbins too large");
    int sms = 148;
    int dev = 0;
    LK_CUDA(cudaGetDevice(&dev));
    LK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    // One block per listed cell up to 32 per SM (blocks past the device-side
    // count exit at once); a block loops over further cells.
    const uint64_t blocks = std::min<uint64_t>(max_cells, static_cast<uint64_t>(sms) * 32);
    auto launch = [&](auto kern) {
        sc::set_smem(kern, smem);
        kern<<<static_cast<unsigned>(blocks), kThreads, smem, s>>>(d_fold0, t, sp, rs, d_cells,
                                                                   d_count, max_cells, d_scores);
    };
    auto by_nw = [&](auto tg) {
        constexpr bool TG = decltype(tg)::value;
        sc::dispatch_nw_nb(sp.nwidths, t.nbins, [&](auto nw, auto nbc) {
            launch(rescore_kernel<TG, decltype(nw)::value, decltype(nbc)::value>);
        });
    };
    if (taylor) {
        by_nw(std::true_type{});
    } else {
        by_nw(std::false_type{});
    }
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
