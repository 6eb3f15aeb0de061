// The pipelined brute-fold kernel (see brute_fold.cu for the design). Kept
// in a header so that each bin count is compiled in its own translation unit
// (brute_fold_nb*.cu): the fully unrolled per-bin replay is large.
#pragma once

#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_ptx.cuh"

namespace lk {
namespace bf {

constexpr int kWarp = 32;
constexpr int kChunk = 128;
constexpr int kStages = 3;

template <int NBINS> constexpr int groups_for() {
    return NBINS <= 32 ? 12 : (NBINS <= 64 ? 8 : 4);
}

// ---- the fold ---------------------------------------------------------------

template <int NBINS, int C, int S, int G>
struct FoldCfg {
    static constexpr int kConsumers = 2 * G;
    static constexpr int kThreads = (kConsumers + 1) * kWarp;
    static constexpr size_t kStageFloats = 2ull * C * kWarp;
    static constexpr size_t kStageBytes = kStageFloats * sizeof(float);
    static constexpr size_t kSmem = S * kStageBytes + 2 * S * sizeof(uint64_t);
};

// Consumer-side pipeline position, shared by the replay helpers below.
struct ReplayState {
    const float* xs;    // ring base
    const float* xrow;  // this warp's row of the current stage, + lane
    uint64_t* full;
    uint64_t* empty;
    uint32_t* status;
    uint32_t il;        // sample index within the current chunk
    uint32_t k;         // current chunk
    uint32_t nchunks;
    uint32_t phase;
    int s;              // current stage
    int row;
    int lane;
};

// Adds the next n samples (in order) to accumulator a, crossing chunk
// boundaries as needed. Returns false if a bounded wait gave up.
template <int C, int S>
__device__ __forceinline__ bool replay_run(float& a, uint32_t n, ReplayState& st) {
    while (n != 0) {
        const uint32_t m = min(n, static_cast<uint32_t>(C) - st.il);
        const float* xp = st.xrow + st.il * kWarp;
        uint32_t t = 0;
        for (; t + 4 <= m; t += 4) {
            const float x0 = xp[(t + 0) * kWarp];
            const float x1 = xp[(t + 1) * kWarp];
            const float x2 = xp[(t + 2) * kWarp];
            const float x3 = xp[(t + 3) * kWarp];
            a = __fadd_rn(a, x0);
            a = __fadd_rn(a, x1);
            a = __fadd_rn(a, x2);
            a = __fadd_rn(a, x3);
        }
        for (; t < m; ++t) {
            a = __fadd_rn(a, xp[t * kWarp]);
        }
        st.il += m;
        n -= m;
        if (st.il == static_cast<uint32_t>(C)) {
            // Every lane releases the stage (release semantics order its
            // reads before the producer's next TMA write into it).
            ptx::mbar_arrive(&st.empty[st.s]);
            ++st.k;
            st.il = 0;
            st.s = (st.s + 1 == S) ? 0 : st.s + 1;
            if (st.s == 0) {
                st.phase ^= 1u;
            }
            st.xrow = st.xs + (static_cast<size_t>(st.s) * 2 + st.row) * C * kWarp + st.lane;
            if (st.k < st.nchunks &&
                !ptx::mbar_wait_bounded(&st.full[st.s], st.phase, st.status,
                                        dev::kStatusWaitTimeout | dev::kStatusFull)) {
                return false;
            }
        }
    }
    return true;
}

// One virtual period: bins Q*8 .. NBINS-1, eight run lengths per 16-byte
// load. Recursion over compile-time bin indices keeps every accumulator in
// a register.
template <int Q, int NBINS, int C, int S>
__device__ __forceinline__ bool replay_period(float (&acc)[NBINS], const uint4* lp,
                                              ReplayState& st) {
    if constexpr (Q * 8 < NBINS) {
        const uint4 w = __ldg(lp + Q);
        if (!replay_run<C, S>(acc[Q * 8 + 0], w.x & 0xffffu, st)) return false;
        if (!replay_run<C, S>(acc[Q * 8 + 1], w.x >> 16, st)) return false;
        if (!replay_run<C, S>(acc[Q * 8 + 2], w.y & 0xffffu, st)) return false;
        if (!replay_run<C, S>(acc[Q * 8 + 3], w.y >> 16, st)) return false;
        if (!replay_run<C, S>(acc[Q * 8 + 4], w.z & 0xffffu, st)) return false;
        if (!replay_run<C, S>(acc[Q * 8 + 5], w.z >> 16, st)) return false;
        if (!replay_run<C, S>(acc[Q * 8 + 6], w.w & 0xffffu, st)) return false;
        if (!replay_run<C, S>(acc[Q * 8 + 7], w.w >> 16, st)) return false;
        return replay_period<Q + 1, NBINS, C, S>(acc, lp, st);
    } else {
        return true;
    }
}

template <int NBINS, int C, int S, int G>
__global__ void __launch_bounds__(FoldCfg<NBINS, C, S, G>::kThreads, 1)
    brute_fold_tma_kernel(const __grid_constant__ CUtensorMap tmap,
                          const uint16_t* __restrict__ lens,
                          const uint64_t* __restrict__ lens_off,
                          const uint32_t* __restrict__ nper, uint32_t nfreq, uint32_t nseg,
                          uint32_t seglen, float* __restrict__ fold, uint32_t* status) {
    using Cfg = FoldCfg<NBINS, C, S, G>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* xs = reinterpret_cast<float*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + S * Cfg::kStageBytes);
    uint64_t* empty = full + S;

    const int warp = threadIdx.x / kWarp;
    const int lane = threadIdx.x % kWarp;
    const uint32_t f0 = blockIdx.y * G;
    const int nactive = static_cast<int>(min(static_cast<uint32_t>(G), nfreq - f0));
    const int nconsumers = 2 * nactive;
    const uint32_t nchunks = seglen / C;

    if (threadIdx.x == 0) {
        ptx::prefetch_tensormap(&tmap);
        for (int s = 0; s < S; ++s) {
            ptx::mbar_init(&full[s], 1);
            ptx::mbar_init(&empty[s], nconsumers * kWarp);
        }
        ptx::fence_barrier_init();
    }
    __syncthreads();

    if (warp == Cfg::kConsumers) {
        // Producer: one thread issues every chunk's TMA load.
        if (lane == 0) {
            uint32_t issued = 0;
            bool ok = true;
            for (uint32_t k = 0; k < nchunks; ++k) {
                const int s = static_cast<int>(k % S);
                if (k >= static_cast<uint32_t>(S)) {
                    ok = ptx::mbar_wait_bounded(&empty[s], ((k / S) - 1) & 1u, status,
                                                dev::kStatusWaitTimeout | dev::kStatusEmpty);
                    if (!ok) {
                        break;
                    }
                }
                ptx::mbar_arrive_expect_tx(&full[s], static_cast<uint32_t>(Cfg::kStageBytes));
                ptx::tma_load_3d(xs + s * Cfg::kStageFloats, &tmap, &full[s],
                                 static_cast<int>(blockIdx.x * kWarp), static_cast<int>(k * C), 0);
                ++issued;
            }
            // Stay resident until the last loads have landed so that no copy
            // is in flight when the block exits (bounded).
            const uint32_t first = issued > static_cast<uint32_t>(S) ? issued - S : 0;
            for (uint32_t k = first; k < issued; ++k) {
                ptx::mbar_wait_bounded(&full[k % S], (k / S) & 1u, status,
                                       dev::kStatusWaitTimeout | dev::kStatusDrain);
            }
        }
        return;
    }
    if (warp >= nconsumers) {
        return;
    }

    const uint32_t f = f0 + static_cast<uint32_t>(warp >> 1);
    const int row = warp & 1;
    const uint16_t* L = lens + lens_off[f];
    const uint32_t np_f = nper[f];

    float acc[NBINS];
#pragma unroll
    for (int b = 0; b < NBINS; ++b) {
        acc[b] = 0.0f;
    }

    ReplayState st;
    st.xs = xs;
    st.xrow = xs + static_cast<size_t>(row) * C * kWarp + lane;
    st.full = full;
    st.empty = empty;
    st.status = status;
    st.il = 0;
    st.k = 0;
    st.nchunks = nchunks;
    st.phase = 0;
    st.s = 0;
    st.row = row;
    st.lane = lane;
    if (!ptx::mbar_wait_bounded(&full[0], 0, status,
                                dev::kStatusWaitTimeout | dev::kStatusFirstFull)) {
        return;
    }
    for (uint32_t p = 0; p < np_f; ++p) {
        const uint4* lp = reinterpret_cast<const uint4*>(L + static_cast<size_t>(p) * NBINS);
        if (!replay_period<0, NBINS, C, S>(acc, lp, st)) {
            return;
        }
    }

    const uint32_t seg = blockIdx.x * kWarp + lane;
    if (seg < nseg) {
        float4* out = reinterpret_cast<float4*>(
            fold + ((static_cast<size_t>(seg) * nfreq + f) * 2 + row) * NBINS);
#pragma unroll
        for (int b = 0; b < NBINS / 4; ++b) {
            out[b] = make_float4(acc[4 * b], acc[4 * b + 1], acc[4 * b + 2], acc[4 * b + 3]);
        }
    }
}


template <int NBINS>
void launch_tma(const CUtensorMap& tmap, const uint16_t* lens, const uint64_t* off,
                const uint32_t* nper, uint32_t nfreq, uint32_t nseg, uint32_t nseg_pad,
                uint32_t seglen, float* fold, uint32_t* status, cudaStream_t s) {
    constexpr int G = groups_for<NBINS>();
    using Cfg = FoldCfg<NBINS, kChunk, kStages, G>;
    auto kern = brute_fold_tma_kernel<NBINS, kChunk, kStages, G>;
    LK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(Cfg::kSmem)));
    dim3 grid(nseg_pad / kWarp, (nfreq + G - 1) / G);
    kern<<<grid, Cfg::kThreads, Cfg::kSmem, s>>>(tmap, lens, off, nper, nfreq, nseg, seglen,
                                                  fold, status);
    LK_CUDA(cudaGetLastError());
}

}  // namespace bf
}  // namespace lk
