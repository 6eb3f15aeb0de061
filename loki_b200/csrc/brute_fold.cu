// Brute fold (level 0 of the FFA) on sm_100a.
//
// out[seg, f, r, b] = sum over samples i of segment seg whose phase bin at
// frequency f is b, of ts_r[seg * seglen + i], added in increasing i starting
// from 0.0f -- the reference's order (lib/fold.cpp:113-142,
// lib/kernels.cpp:550-580,1132-1154), so results are bit-identical.
//
// Plan-time tables (host, once per plan): the sample -> bin map of one
// segment is the same for every segment. For each frequency it is encoded as
//   * one 32-bit word per 32 samples whose bit i is set when sample i starts
//     a run of equal bin (the bin differs from the previous sample's), and
//   * the bin of every run, in sample order (uint8, or uint16 for nbins > 256).
//
// Execution (one block = 32 segments x W frequencies):
//  * a producer thread streams 32-sample words of the 32 segments, E and V
//    rows, straight from the series with 2-D TMA loads into a shared-memory
//    ring; the tiles use the 128-byte swizzle, so lane l (segment l) reads its
//    own 32 consecutive samples of a row with eight conflict-free 16-byte
//    loads;
//  * each consumer warp owns one frequency and both rows (E and V share the
//    run mask): per word it walks the samples in registers (fully unrolled)
//    four at a time -- a group without a run start is four adds per row --
//    and at each run start stores the running sums to the bin's accumulators
//    ([row][bin][lane] in shared memory, conflict-free), fetches the next
//    run's bin by warp shuffle and reloads that bin's accumulators. All lanes
//    follow the same mask, so control flow is uniform.
//
// Packed form (both rows per warp, the default for nbins <= 64): the series
// is first interleaved into (e, v) pairs, so one 16-byte shared-memory load
// yields two samples' pairs in adjacent registers and each sample is one
// add.rn.f32x2 (two IEEE round-to-nearest adds, E and V, in one
// instruction); accumulators are float2 [bin][lane]. Measured on B200
// (2^22-sample accelerated workload, nbins 64): 1.95 ms against 2.23 ms for
// two scalar adds. Loading the next run's sums one run ahead measured slower
// here too (2.07 ms); for nbins 128 one row per warp stays faster (7.39
// against 7.71 ms on the 2^21-sample frequency sweep). Two frequencies per
// warp sharing the sample registers (3.51 ms, half the warps fit) and each
// frequency's bins split over two or four warps that skip words outside
// their bins (2.55 / 3.64 ms) were slower as well. Frequencies whose bins step
// by one at every run (every frequency below 1 / (tsamp nbins)) take a path
// without the bin table, with the next run's sums loaded a run ahead (1.82
// ms); dispatching each four-sample group through a 16-way switch instead of
// per-sample run-start tests measured slower (2.46 ms). With tensor-memory
// sums (below; 1.58 ms), two 32-segment groups per warp sharing one
// frequency's run handling (two add chains per warp, float4 sums, at most 13
// warps) measured slower as well: 2.41 ms at best. Reading separate E and V
// tiles and pairing them in registers (no interleave pass, 0.019 ms saved)
// made the fold itself 1.79 ms against 1.57 ms: the interleave pass stays.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <type_traits>

#include <cudaTypedefs.h>

#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_ptx.cuh"

namespace lk {

namespace {

constexpr int kWarp = 32;
constexpr int kMaxStages = 16;
constexpr uint32_t kTileBytes = 32 * 32 * sizeof(float);  // 32 samples x 32 segments
constexpr uint32_t kStageBytes = 2 * kTileBytes;           // E and V rows, 8 KiB
constexpr size_t kSmemLimit = 227 * 1024;
constexpr int kMaxConsumers = 19;  // + 1 producer warp = 640 threads (<= 102 registers)

// Host restatement of psr_utils::get_phase_idx_uint
// (lib/loki/psr_utils.hpp:32-63): IEEE double, no contraction.
uint32_t host_phase_bin(double proper_time, double freq, uint64_t nbins) {
    const double total_phase = (proper_time - 0.0) * freq;
    const double norm_phase = total_phase - std::floor(total_phase);
    double iphase = norm_phase * static_cast<double>(nbins);
    if (iphase >= static_cast<double>(nbins)) {
        iphase = 0.0;
    }
    const auto f = static_cast<float>(iphase);
    auto b = static_cast<uint32_t>(f + 0.5F);
    return b == nbins ? 0u : b;
}

struct FoldArgs {
    const uint32_t* masks;     // [nfreq][nwords] run-start bits
    const void* bins;          // run bins of all frequencies (uint8 or uint16)
    const uint64_t* bin_off;   // first run of each frequency
    const uint64_t* nruns;     // runs of each frequency
    const uint8_t* seq;        // 1: frequency's run bins go b, b+1, b+2, ... (mod nbins)
    uint32_t nfreq;
    uint32_t nseg;
    uint32_t nbins;
    uint32_t nwords;           // ceil(seglen / 32)
    uint32_t warps;            // W consumer warps (frequencies) per block
    uint32_t smem_warps;       // TMEM kernel: consumers with shared-memory sums (the rest use TMEM)
    uint32_t stages;           // depth of the shared-memory ring (<= kMaxStages)
    float* fold;
    uint32_t* status;
    // Segment-group mode (packed kernels, batches of zero-padded series):
    // block b folds the 32 segments of groups 4 b .. 4 b + 3, each group 8
    // consecutive segments starting at row groups[g]; blocks with 4 b >=
    // *ngroups have no work. nullptr: block b folds segments 32 b .. 32 b + 31.
    const uint32_t* groups;
    const uint32_t* ngroups;
};

// Group mode: true when the block has at least one segment group.
__device__ __forceinline__ bool block_has_groups(const FoldArgs& a) {
    return blockIdx.x * 4u < *a.ngroups;
}

// Group mode: the first rows of the block's four groups (a missing group
// re-reads the block's first group; its lanes do not store).
__device__ __forceinline__ void block_group_rows(const FoldArgs& a, uint32_t (&grow)[4]) {
    const uint32_t ng = *a.ngroups;
    const uint32_t g0 = blockIdx.x * 4u;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        grow[q] = a.groups[g0 + q < ng ? g0 + q : g0];
    }
}

// The segment whose fold lane `lane` holds, and whether it is stored.
__device__ __forceinline__ uint32_t lane_segment(const FoldArgs& a, int seg0, int lane, bool* store) {
    if (a.groups == nullptr) {
        const auto seg = static_cast<uint32_t>(seg0 + lane);
        *store = seg < a.nseg;
        return seg;
    }
    const uint32_t g = blockIdx.x * 4u + static_cast<uint32_t>(lane / 8);
    *store = g < *a.ngroups;
    return a.groups[*store ? g : blockIdx.x * 4u] + static_cast<uint32_t>(lane % 8);
}

// One word's two 32-float boxes of (e, v) pairs into a stage: 32 rows from
// seg0, or (group mode) four 8-row boxes, each into its 1024-byte quarter of
// the tile, where the 128-byte swizzle of rows 8 q .. 8 q + 7 is the same.
__device__ __forceinline__ void load_word(unsigned char* st, const CUtensorMap* tmap_ev,
                                          const CUtensorMap* tmap_ev8, uint64_t* bar, int x0,
                                          int seg0, bool grouped, const uint32_t (&grow)[4]) {
    if (!grouped) {
        ptx::tma_load_2d(st, tmap_ev, bar, x0, seg0);
        ptx::tma_load_2d(st + kTileBytes, tmap_ev, bar, x0 + 32, seg0);
        return;
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            ptx::tma_load_2d(st + h * kTileBytes + q * 1024, tmap_ev8, bar, x0 + 32 * h,
                             static_cast<int>(grow[q]));
        }
    }
}

template <class BinT>
__device__ __forceinline__ uint32_t load_bins(const BinT* b, uint64_t n, uint64_t first,
                                              int lane) {
    const uint64_t k = first + static_cast<uint64_t>(lane);
    return k < n ? static_cast<uint32_t>(__ldg(b + k)) : 0u;
}

// ROWS = 2: a consumer warp owns one frequency and both rows (E and V share
// the run mask and run bins); ROWS = 1: one (frequency, row) item per warp,
// half the accumulator memory per warp, so twice the warps fit a block
// (used for large nbins, where accumulators limit the warps per SM).
template <class BinT, int ROWS>
__global__ void __launch_bounds__(640, 1)
    brute_fold_mask_kernel(const __grid_constant__ CUtensorMap tmap_e,
                           const __grid_constant__ CUtensorMap tmap_v, FoldArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // Stages first (1024-byte aligned for the 128-byte swizzle), then the
    // barriers, then the accumulators.
    const uint32_t S = a.stages;
    unsigned char* ring = smem_raw;
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + S * kStageBytes);
    uint64_t* empty = full + S;
    float* accs = reinterpret_cast<float*>(empty + S);

    const int warp = threadIdx.x / kWarp;
    const int lane = threadIdx.x % kWarp;
    const int W = static_cast<int>(a.warps);
    const uint32_t q0 = blockIdx.y * a.warps;  // first work item of the block
    const uint32_t nitems = (ROWS == 2 ? 1u : 2u) * a.nfreq;
    const int nconsumers = static_cast<int>(min(a.warps, nitems - q0));
    const int seg0 = static_cast<int>(blockIdx.x * kWarp);

    // The 128-byte swizzle pattern is defined on 1024-byte aligned tiles.
    if ((ptx::smem_u32(ring) & 1023u) != 0) {
        if (threadIdx.x == 0) {
            atomicOr(a.status, dev::kStatusBadTable);
        }
        return;
    }
    if (threadIdx.x == 0) {
        ptx::prefetch_tensormap(&tmap_e);
        ptx::prefetch_tensormap(&tmap_v);
        for (uint32_t s = 0; s < S; ++s) {
            ptx::mbar_init(&full[s], 1);
            ptx::mbar_init(&empty[s], nconsumers * kWarp);
        }
        ptx::fence_barrier_init();
    }
    __syncthreads();

    if (warp == W) {
        // Producer: one thread issues each 32-sample word's E and V tiles.
        if (lane == 0) {
            uint32_t issued = 0;
            for (uint32_t k = 0; k < a.nwords; ++k) {
                const uint32_t s = k % S;
                if (k >= S &&
                    !ptx::mbar_wait_bounded(&empty[s], ((k / S) - 1) & 1u, a.status,
                                            dev::kStatusWaitTimeout | dev::kStatusEmpty)) {
                    break;
                }
                unsigned char* st = ring + static_cast<size_t>(s) * kStageBytes;
                ptx::mbar_arrive_expect_tx(&full[s], kStageBytes);
                const int x0 = static_cast<int>(k * 32);
                ptx::tma_load_2d(st, &tmap_e, &full[s], x0, seg0);
                ptx::tma_load_2d(st + kTileBytes, &tmap_v, &full[s], x0, seg0);
                ++issued;
            }
            // Stay resident until the last loads have landed (bounded).
            const uint32_t first = issued > S ? issued - S : 0;
            for (uint32_t k = first; k < issued; ++k) {
                ptx::mbar_wait_bounded(&full[k % S], (k / S) & 1u, a.status,
                                       dev::kStatusWaitTimeout | dev::kStatusDrain);
            }
        }
        return;
    }
    if (warp >= nconsumers) {
        return;
    }

    const uint32_t q = q0 + static_cast<uint32_t>(warp);
    const uint32_t f = ROWS == 2 ? q : (q >> 1);
    const uint32_t row0 = ROWS == 2 ? 0u : (q & 1u);
    // Accumulators of this warp: ROWS rows of [nbins + 1][32 lanes]; slot
    // nbins is a scratch slot that absorbs the store before the first run.
    const uint32_t vrow = (a.nbins + 1) * kWarp;
    float* A = accs + static_cast<size_t>(warp) * ROWS * vrow + lane;
    for (uint32_t b = 0; b < ROWS * (a.nbins + 1); ++b) {
        A[b * kWarp] = 0.0f;
    }
    const uint32_t* M = a.masks + static_cast<size_t>(f) * a.nwords;
    const BinT* B = static_cast<const BinT*>(a.bins) + a.bin_off[f];
    const uint64_t nr = a.nruns[f];
    // Swizzled tile offset of lane l's 16-byte chunk j: l*128 + ((j ^ (l & 7)) * 16).
    const uint32_t lrow = static_cast<uint32_t>(lane) * 128u;
    const uint32_t lsw = static_cast<uint32_t>(lane) & 7u;

    // The word loop; SEQ as in the packed kernel (run bins step by one: no
    // table, next run's sums loaded a run ahead).
    auto consume = [&](auto seq_tag) -> bool {
        constexpr bool SEQ = decltype(seq_tag)::value;
        uint32_t bin;
        float acc0 = 0.0f, acc1 = 0.0f;
        float nacc0 = 0.0f, nacc1 = 0.0f;  // SEQ: sums of bin + 1
        uint64_t r = 0;      // runs started so far
        uint64_t rbase = 0;  // run index held by lane 0 of binbuf
        uint32_t binbuf = 0;
        if constexpr (SEQ) {
            const uint32_t b0 = static_cast<uint32_t>(__ldg(B));
            bin = b0 == 0 ? a.nbins - 1 : b0 - 1;
        } else {
            bin = a.nbins;  // scratch slot before the first run
            binbuf = load_bins(B, nr, 0, lane);
        }
        uint32_t maskbuf = __ldg(M + min(static_cast<uint32_t>(lane), a.nwords - 1));

        // Starts run rl (relative to rbase): flush the current sums, move to
        // the run's bin and its sums.
        auto start_run = [&](uint32_t& rl) {
            A[bin * kWarp] = acc0;
            if constexpr (ROWS == 2) {
                A[vrow + bin * kWarp] = acc1;
            }
            if constexpr (SEQ) {
                bin = bin + 1 == a.nbins ? 0u : bin + 1;
                acc0 = nacc0;
                acc1 = nacc1;
                const uint32_t nb = bin + 1 == a.nbins ? 0u : bin + 1;
                nacc0 = A[nb * kWarp];
                if constexpr (ROWS == 2) {
                    nacc1 = A[vrow + nb * kWarp];
                }
                ++rl;
            } else {
                bin = __shfl_sync(0xffffffffu, binbuf, static_cast<int>(rl));
                ++rl;
                acc0 = A[bin * kWarp];
                if constexpr (ROWS == 2) {
                    acc1 = A[vrow + bin * kWarp];
                }
            }
        };

        uint32_t phase = 0;
        uint32_t s = 0;
        for (uint32_t c = 0; c < a.nwords; ++c) {
            if ((c & 31u) == 0 && c > 0) {
                maskbuf = __ldg(M + min(c + static_cast<uint32_t>(lane), a.nwords - 1));
            }
            const uint32_t m = __shfl_sync(0xffffffffu, maskbuf, static_cast<int>(c & 31u));
            if constexpr (!SEQ) {
                // binbuf must hold runs r .. r + popc(m) - 1.
                if (r + static_cast<uint64_t>(__popc(m)) > rbase + 32) {
                    rbase = r;
                    binbuf = load_bins(B, nr, rbase, lane);
                }
            }
            if (!ptx::mbar_wait_bounded(&full[s], phase, a.status,
                                        dev::kStatusWaitTimeout |
                                            (c == 0 ? dev::kStatusFirstFull : dev::kStatusFull))) {
                return false;
            }
            const unsigned char* te =
                ring + static_cast<size_t>(s) * kStageBytes + row0 * kTileBytes + lrow;
            float x0[32];
            [[maybe_unused]] float x1[ROWS == 2 ? 32 : 1];
#pragma unroll
            for (uint32_t j = 0; j < 8; ++j) {
                const uint32_t o = (j ^ lsw) << 4;
                const float4 v0 = *reinterpret_cast<const float4*>(te + o);
                x0[4 * j + 0] = v0.x;
                x0[4 * j + 1] = v0.y;
                x0[4 * j + 2] = v0.z;
                x0[4 * j + 3] = v0.w;
                if constexpr (ROWS == 2) {
                    const float4 v1 = *reinterpret_cast<const float4*>(te + kTileBytes + o);
                    x1[4 * j + 0] = v1.x;
                    x1[4 * j + 1] = v1.y;
                    x1[4 * j + 2] = v1.z;
                    x1[4 * j + 3] = v1.w;
                }
            }
            // Release the stage as soon as its samples are in registers.
            ptx::mbar_arrive(&empty[s]);
            s = (s + 1 == S) ? 0 : s + 1;
            if (s == 0) {
                phase ^= 1u;
            }
            uint32_t rl = static_cast<uint32_t>(r - rbase);
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                if (((m >> (4 * g)) & 0xfu) == 0) {
#pragma unroll
                    for (int i = 4 * g; i < 4 * g + 4; ++i) {
                        acc0 = __fadd_rn(acc0, x0[i]);
                        if constexpr (ROWS == 2) {
                            acc1 = __fadd_rn(acc1, x1[i]);
                        }
                    }
                } else {
#pragma unroll
                    for (int i = 4 * g; i < 4 * g + 4; ++i) {
                        if (m & (1u << i)) {
                            start_run(rl);
                        }
                        acc0 = __fadd_rn(acc0, x0[i]);
                        if constexpr (ROWS == 2) {
                            acc1 = __fadd_rn(acc1, x1[i]);
                        }
                    }
                }
            }
            r = rbase + rl;
        }
        A[bin * kWarp] = acc0;
        if constexpr (ROWS == 2) {
            A[vrow + bin * kWarp] = acc1;
        }
        if (r != nr) {
            atomicOr(a.status, dev::kStatusBadTable);
        }
        return true;
    };
    const bool ok = a.seq[f] != 0 ? consume(std::true_type{}) : consume(std::false_type{});
    if (!ok) {
        return;
    }

    const uint32_t seg = static_cast<uint32_t>(seg0 + lane);
    if (seg < a.nseg) {
#pragma unroll
        for (int k = 0; k < ROWS; ++k) {
            const float* R = A + k * vrow;
            const uint32_t row = row0 + static_cast<uint32_t>(k);
            float* out = a.fold + ((static_cast<size_t>(seg) * a.nfreq + f) * 2 + row) * a.nbins;
            if ((a.nbins & 3u) == 0) {
                for (uint32_t b = 0; b < a.nbins; b += 4) {
                    reinterpret_cast<float4*>(out)[b / 4] = make_float4(
                        R[b * kWarp], R[(b + 1) * kWarp], R[(b + 2) * kWarp], R[(b + 3) * kWarp]);
                }
            } else {
                for (uint32_t b = 0; b < a.nbins; ++b) {
                    out[b] = R[b * kWarp];
                }
            }
        }
    }
}

// Two IEEE round-to-nearest FP32 adds (a.x + b.x, a.y + b.y) in one sm_100a
// instruction; bit-identical to two __fadd_rn.
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) {
    uint64_t ra, rb, rd;
    asm("mov.b64 %0, {%1, %2};" : "=l"(ra) : "f"(a.x), "f"(a.y));
    asm("mov.b64 %0, {%1, %2};" : "=l"(rb) : "f"(b.x), "f"(b.y));
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(rd));
    return r;
}

// Packed form: one frequency and both rows per consumer warp, input tiles of
// (e, v) pairs. Same pipeline, tables and order of adds as the mask kernel.
template <class BinT>
__global__ void __launch_bounds__(640, 1)
    brute_fold_pk_kernel(const __grid_constant__ CUtensorMap tmap_ev,
                         const __grid_constant__ CUtensorMap tmap_ev8, FoldArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const bool grouped = a.groups != nullptr;
    if (grouped && !block_has_groups(a)) {
        return;  // uniform: no group for this block
    }
    const uint32_t S = a.stages;
    unsigned char* ring = smem_raw;
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + S * kStageBytes);
    uint64_t* empty = full + S;
    float2* accs = reinterpret_cast<float2*>(empty + S);

    const int warp = threadIdx.x / kWarp;
    const int lane = threadIdx.x % kWarp;
    const int W = static_cast<int>(a.warps);
    // A block folds W consecutive frequencies: the warps share the sample
    // ring and so move at the pace of the slowest, and neighbouring
    // frequencies have nearly the same number of run starts. (Dealing the
    // frequencies round-robin over the blocks put a high frequency in every
    // block and measured 30 % slower.)
    const uint32_t q0 = blockIdx.y * a.warps;
    const int nconsumers = static_cast<int>(min(a.warps, a.nfreq - q0));
    const int seg0 = static_cast<int>(blockIdx.x * kWarp);

    if ((ptx::smem_u32(ring) & 1023u) != 0) {
        if (threadIdx.x == 0) {
            atomicOr(a.status, dev::kStatusBadTable);
        }
        return;
    }
    if (threadIdx.x == 0) {
        ptx::prefetch_tensormap(grouped ? &tmap_ev8 : &tmap_ev);
        for (uint32_t s = 0; s < S; ++s) {
            ptx::mbar_init(&full[s], 1);
            ptx::mbar_init(&empty[s], nconsumers * kWarp);
        }
        ptx::fence_barrier_init();
    }
    __syncthreads();

    if (warp == W) {
        // Producer: word k is samples 32k .. 32k+31, i.e. floats 64k ..
        // 64k+63 of each segment's interleaved row, as two 32-float boxes
        // (eight 8-row boxes in group mode).
        if (lane == 0) {
            uint32_t grow[4] = {0, 0, 0, 0};
            if (grouped) {
                block_group_rows(a, grow);
            }
            uint32_t issued = 0;
            for (uint32_t k = 0; k < a.nwords; ++k) {
                const uint32_t s = k % S;
                if (k >= S &&
                    !ptx::mbar_wait_bounded(&empty[s], ((k / S) - 1) & 1u, a.status,
                                            dev::kStatusWaitTimeout | dev::kStatusEmpty)) {
                    break;
                }
                unsigned char* st = ring + static_cast<size_t>(s) * kStageBytes;
                ptx::mbar_arrive_expect_tx(&full[s], kStageBytes);
                load_word(st, &tmap_ev, &tmap_ev8, &full[s], static_cast<int>(k * 64), seg0, grouped,
                          grow);
                ++issued;
            }
            const uint32_t first = issued > S ? issued - S : 0;
            for (uint32_t k = first; k < issued; ++k) {
                ptx::mbar_wait_bounded(&full[k % S], (k / S) & 1u, a.status,
                                       dev::kStatusWaitTimeout | dev::kStatusDrain);
            }
        }
        return;
    }
    if (warp >= nconsumers) {
        return;
    }

    const uint32_t f = q0 + static_cast<uint32_t>(warp);
    // [nbins + 1][32 lanes] (E, V) sums; slot nbins absorbs the store before
    // the first run.
    float2* A = accs + static_cast<size_t>(warp) * (a.nbins + 1) * kWarp + lane;
    for (uint32_t b = 0; b <= a.nbins; ++b) {
        A[b * kWarp] = make_float2(0.0f, 0.0f);
    }
    const uint32_t* M = a.masks + static_cast<size_t>(f) * a.nwords;
    const BinT* B = static_cast<const BinT*>(a.bins) + a.bin_off[f];
    const uint64_t nr = a.nruns[f];
    const uint32_t lrow = static_cast<uint32_t>(lane) * 128u;
    const uint32_t lsw = static_cast<uint32_t>(lane) & 7u;

    // The word loop, for SEQ = run bins b, b+1, ... (mod nbins) or any order.
    // SEQ: a run's bin is the previous one plus one, so no table read, and the
    // next run's sums are loaded as soon as a run starts (the only store before
    // they are used is the current bin's, and the next bin differs from it),
    // which takes the load off the add chain. Other frequencies read each
    // run's bin from the table by warp shuffle.
    auto consume = [&](auto seq_tag) -> bool {
        constexpr bool SEQ = decltype(seq_tag)::value;
        uint32_t bin;
        float2 acc = make_float2(0.0f, 0.0f);
        float2 nacc = make_float2(0.0f, 0.0f);  // SEQ: sums of bin + 1
        uint64_t r = 0;
        uint64_t rbase = 0;
        uint32_t binbuf = 0;
        if constexpr (SEQ) {
            // The first run (sample 0) starts at bin b0: begin "before" it at
            // b0 - 1, whose sums are still zero, so the first run start
            // stores a zero there and moves to b0 with zero sums.
            const uint32_t b0 = static_cast<uint32_t>(__ldg(B));
            bin = b0 == 0 ? a.nbins - 1 : b0 - 1;
        } else {
            bin = a.nbins;  // scratch slot before the first run
            binbuf = load_bins(B, nr, 0, lane);
        }
        uint32_t maskbuf = __ldg(M + min(static_cast<uint32_t>(lane), a.nwords - 1));

        auto start_run = [&](uint32_t& rl) {
            A[bin * kWarp] = acc;
            if constexpr (SEQ) {
                bin = bin + 1 == a.nbins ? 0u : bin + 1;
                acc = nacc;
                const uint32_t nb = bin + 1 == a.nbins ? 0u : bin + 1;
                nacc = A[nb * kWarp];
                ++rl;
            } else {
                bin = __shfl_sync(0xffffffffu, binbuf, static_cast<int>(rl));
                ++rl;
                acc = A[bin * kWarp];
            }
        };

        uint32_t phase = 0;
        uint32_t s = 0;
        for (uint32_t c = 0; c < a.nwords; ++c) {
            if ((c & 31u) == 0 && c > 0) {
                maskbuf = __ldg(M + min(c + static_cast<uint32_t>(lane), a.nwords - 1));
            }
            const uint32_t m = __shfl_sync(0xffffffffu, maskbuf, static_cast<int>(c & 31u));
            if constexpr (!SEQ) {
                if (r + static_cast<uint64_t>(__popc(m)) > rbase + 32) {
                    rbase = r;
                    binbuf = load_bins(B, nr, rbase, lane);
                }
            }
            if (!ptx::mbar_wait_bounded(&full[s], phase, a.status,
                                        dev::kStatusWaitTimeout |
                                            (c == 0 ? dev::kStatusFirstFull : dev::kStatusFull))) {
                return false;
            }
            const unsigned char* t0 = ring + static_cast<size_t>(s) * kStageBytes + lrow;
            float2 x[32];
#pragma unroll
            for (uint32_t h = 0; h < 2; ++h) {
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j) {
                    const uint32_t o = (j ^ lsw) << 4;
                    const float4 v = *reinterpret_cast<const float4*>(t0 + h * kTileBytes + o);
                    x[16 * h + 2 * j] = make_float2(v.x, v.y);
                    x[16 * h + 2 * j + 1] = make_float2(v.z, v.w);
                }
            }
            ptx::mbar_arrive(&empty[s]);
            s = (s + 1 == S) ? 0 : s + 1;
            if (s == 0) {
                phase ^= 1u;
            }
            uint32_t rl = static_cast<uint32_t>(r - rbase);
#pragma unroll
            for (int g = 0; g < 8; ++g) {
                if (((m >> (4 * g)) & 0xfu) == 0) {
#pragma unroll
                    for (int i = 4 * g; i < 4 * g + 4; ++i) {
                        acc = add2_rn(acc, x[i]);
                    }
                } else {
#pragma unroll
                    for (int i = 4 * g; i < 4 * g + 4; ++i) {
                        if (m & (1u << i)) {
                            start_run(rl);
                        }
                        acc = add2_rn(acc, x[i]);
                    }
                }
            }
            r = rbase + rl;
        }
        A[bin * kWarp] = acc;
        if (r != nr) {
            atomicOr(a.status, dev::kStatusBadTable);
        }
        return true;
    };
    const bool ok = a.seq[f] != 0 ? consume(std::true_type{}) : consume(std::false_type{});
    if (!ok) {
        return;
    }

    bool store;
    const uint32_t seg = lane_segment(a, seg0, lane, &store);
    if (store) {
        float* out = a.fold + (static_cast<size_t>(seg) * a.nfreq + f) * 2 * a.nbins;
        if ((a.nbins & 3u) == 0) {
            for (uint32_t b = 0; b < a.nbins; b += 4) {
                const float2 p0 = A[b * kWarp], p1 = A[(b + 1) * kWarp];
                const float2 p2 = A[(b + 2) * kWarp], p3 = A[(b + 3) * kWarp];
                reinterpret_cast<float4*>(out)[b / 4] = make_float4(p0.x, p1.x, p2.x, p3.x);
                reinterpret_cast<float4*>(out + a.nbins)[b / 4] =
                    make_float4(p0.y, p1.y, p2.y, p3.y);
            }
        } else {
            for (uint32_t b = 0; b < a.nbins; ++b) {
                const float2 p = A[b * kWarp];
                out[b] = p.x;
                out[a.nbins + b] = p.y;
            }
        }
    }
}

// Packed form with part of the accumulators in tensor memory. The block's
// first a.smem_warps consumer warps keep their float2 [bin][lane] sums in
// shared memory as in brute_fold_pk_kernel; the next consumer warps keep
// them in TMEM (each lane's sums in its TMEM lane: column 2 b holds bin b's
// E sum, 2 b + 1 its V sum), so a block runs more frequencies than shared
// memory alone holds. Every add is the same add.rn.f32x2 in the same order.
// The TMEM ops of a warp are warp-collective: the run masks are shared by
// all lanes, so control flow is uniform, and a timed-out wait makes the
// whole warp stop (__all_sync). TMEM order: a run-ahead read is waited for
// before its sums are used; stores are waited for at every word (a bin is
// revisited only after nbins runs, >= 64 samples when nbins >= 64) and before
// every read when nbins < 64 or the bins do not step by one.
// The producer warp allocates all 512 columns and frees them after the final
// barrier, which every warp reaches (no early return).
constexpr uint32_t kTmemCols = 512;
constexpr int kMaxWarpsTm = 25;  // consumers + producer (<= 72 registers)

template <class BinT>
__global__ void __launch_bounds__(kMaxWarpsTm * 32, 1)
    brute_fold_pk_tm_kernel(const __grid_constant__ CUtensorMap tmap_ev,
                            const __grid_constant__ CUtensorMap tmap_ev8, FoldArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const bool grouped = a.groups != nullptr;
    if (grouped && !block_has_groups(a)) {
        return;  // uniform, before any tensor memory is allocated
    }
    const uint32_t S = a.stages;
    unsigned char* ring = smem_raw;
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + S * kStageBytes);
    uint64_t* empty = full + S;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(empty + S);
    float2* accs = reinterpret_cast<float2*>(tslot + 2);  // 8-byte aligned

    const int warp = threadIdx.x / kWarp;
    const int lane = threadIdx.x % kWarp;
    const int W = static_cast<int>(a.warps);
    const int WS = static_cast<int>(a.smem_warps);
    // W consecutive frequencies per block, as in brute_fold_pk_kernel; the
    // TMEM warps take the block's first slots, its lowest frequencies (the
    // fewest run starts, whose TMEM round trips cost the most).
    const uint32_t q0 = blockIdx.y * a.warps;
    const int nconsumers = static_cast<int>(min(a.warps, a.nfreq - q0));
    const int slot = warp >= WS ? warp - WS : warp + (W - WS);
    const int seg0 = static_cast<int>(blockIdx.x * kWarp);
    const bool aligned = (ptx::smem_u32(ring) & 1023u) == 0;

    if (warp == W) {
        ptx::tmem_alloc(tslot, kTmemCols);
        __syncwarp();
        ptx::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        if (!aligned) {
            atomicOr(a.status, dev::kStatusBadTable);
        }
        ptx::prefetch_tensormap(grouped ? &tmap_ev8 : &tmap_ev);
        for (uint32_t s = 0; s < S; ++s) {
            ptx::mbar_init(&full[s], 1);
            ptx::mbar_init(&empty[s], nconsumers * kWarp);
        }
        ptx::fence_barrier_init();
    }
    ptx::tmem_fence_before_sync();
    __syncthreads();
    ptx::tmem_fence_after_sync();
    const uint32_t tbase = *tslot;

    if (aligned && warp == W) {
        if (lane == 0) {
            uint32_t grow[4] = {0, 0, 0, 0};
            if (grouped) {
                block_group_rows(a, grow);
            }
            uint32_t issued = 0;
            for (uint32_t k = 0; k < a.nwords; ++k) {
                const uint32_t s = k % S;
                if (k >= S &&
                    !ptx::mbar_wait_bounded(&empty[s], ((k / S) - 1) & 1u, a.status,
                                            dev::kStatusWaitTimeout | dev::kStatusEmpty)) {
                    break;
                }
                unsigned char* st = ring + static_cast<size_t>(s) * kStageBytes;
                ptx::mbar_arrive_expect_tx(&full[s], kStageBytes);
                load_word(st, &tmap_ev, &tmap_ev8, &full[s], static_cast<int>(k * 64), seg0, grouped,
                          grow);
                ++issued;
            }
            const uint32_t first = issued > S ? issued - S : 0;
            for (uint32_t k = first; k < issued; ++k) {
                ptx::mbar_wait_bounded(&full[k % S], (k / S) & 1u, a.status,
                                       dev::kStatusWaitTimeout | dev::kStatusDrain);
            }
        }
    } else if (aligned && warp < W && slot < nconsumers) {
        const bool tm = warp >= WS;
        const uint32_t f = q0 + static_cast<uint32_t>(slot);
        // shared-memory sums: [nbins + 1][32 lanes]; slot nbins absorbs the
        // store before the first run. TMEM sums: this warp's quadrant, column
        // block (warp - WS) / 4.
        float2* A = accs + static_cast<size_t>(tm ? 0 : warp) * (a.nbins + 1) * kWarp + lane;
        const uint32_t T = tbase + ((static_cast<uint32_t>(warp & 3) * 32u) << 16) +
                           static_cast<uint32_t>((warp - WS) / 4) * 2u * a.nbins;
        if (tm) {
            for (uint32_t b = 0; b < a.nbins; ++b) {
                ptx::tmem_st2(T + 2 * b, 0.0f, 0.0f);
            }
            ptx::tmem_wait_st();
        } else {
            for (uint32_t b = 0; b <= a.nbins; ++b) {
                A[b * kWarp] = make_float2(0.0f, 0.0f);
            }
        }
        const uint32_t* M = a.masks + static_cast<size_t>(f) * a.nwords;
        const BinT* B = static_cast<const BinT*>(a.bins) + a.bin_off[f];
        const uint64_t nr = a.nruns[f];
        const uint32_t lrow = static_cast<uint32_t>(lane) * 128u;
        const uint32_t lsw = static_cast<uint32_t>(lane) & 7u;

        auto consume = [&](auto seq_tag, auto tm_tag) -> bool {
            constexpr bool SEQ = decltype(seq_tag)::value;
            constexpr bool TM = decltype(tm_tag)::value;
            uint32_t bin;
            float2 acc = make_float2(0.0f, 0.0f);
            float2 nacc = make_float2(0.0f, 0.0f);
            uint64_t r = 0;
            uint64_t rbase = 0;
            uint32_t binbuf = 0;
            if constexpr (SEQ) {
                const uint32_t b0 = static_cast<uint32_t>(__ldg(B));
                bin = b0 == 0 ? a.nbins - 1 : b0 - 1;
            } else {
                bin = a.nbins;
                binbuf = load_bins(B, nr, 0, lane);
            }
            uint32_t maskbuf = __ldg(M + min(static_cast<uint32_t>(lane), a.nwords - 1));
            const bool small = a.nbins < 64;

            auto start_run = [&](uint32_t& rl) {
                if constexpr (TM) {
                    if (SEQ || bin != a.nbins) {
                        ptx::tmem_st2(T + 2 * bin, acc.x, acc.y);
                    }
                } else {
                    A[bin * kWarp] = acc;
                }
                if constexpr (SEQ) {
                    bin = bin + 1 == a.nbins ? 0u : bin + 1;
                    if constexpr (TM) {
                        ptx::tmem_wait_ld(nacc.x, nacc.y);
                    }
                    acc = nacc;
                    const uint32_t nb = bin + 1 == a.nbins ? 0u : bin + 1;
                    if constexpr (TM) {
                        if (small) {
                            ptx::tmem_wait_st();
                        }
                        ptx::tmem_ld2(T + 2 * nb, nacc.x, nacc.y);
                    } else {
                        nacc = A[nb * kWarp];
                    }
                    ++rl;
                } else {
                    bin = __shfl_sync(0xffffffffu, binbuf, static_cast<int>(rl));
                    ++rl;
                    if constexpr (TM) {
                        ptx::tmem_wait_st();
                        ptx::tmem_ld2(T + 2 * bin, acc.x, acc.y);
                        ptx::tmem_wait_ld(acc.x, acc.y);
                    } else {
                        acc = A[bin * kWarp];
                    }
                }
            };

            uint32_t phase = 0;
            uint32_t s = 0;
            for (uint32_t c = 0; c < a.nwords; ++c) {
                if ((c & 31u) == 0 && c > 0) {
                    maskbuf = __ldg(M + min(c + static_cast<uint32_t>(lane), a.nwords - 1));
                }
                const uint32_t m = __shfl_sync(0xffffffffu, maskbuf, static_cast<int>(c & 31u));
                if constexpr (!SEQ) {
                    if (r + static_cast<uint64_t>(__popc(m)) > rbase + 32) {
                        rbase = r;
                        binbuf = load_bins(B, nr, rbase, lane);
                    }
                }
                const bool got = ptx::mbar_wait_bounded(
                    &full[s], phase, a.status,
                    dev::kStatusWaitTimeout | (c == 0 ? dev::kStatusFirstFull : dev::kStatusFull));
                if (!__all_sync(0xffffffffu, got)) {
                    return false;
                }
                if constexpr (TM) {
                    ptx::tmem_wait_st();
                }
                const unsigned char* t0 = ring + static_cast<size_t>(s) * kStageBytes + lrow;
                uint32_t rl = static_cast<uint32_t>(r - rbase);
                // the word in two halves of 16 samples (fewer registers, so
                // more warps fit)
#pragma unroll
                for (uint32_t h = 0; h < 2; ++h) {
                    float2 x[16];
#pragma unroll
                    for (uint32_t j = 0; j < 8; ++j) {
                        const uint32_t o = (j ^ lsw) << 4;
                        const float4 v = *reinterpret_cast<const float4*>(t0 + h * kTileBytes + o);
                        x[2 * j] = make_float2(v.x, v.y);
                        x[2 * j + 1] = make_float2(v.z, v.w);
                    }
                    if (h == 1) {
                        ptx::mbar_arrive(&empty[s]);
                    }
                    const uint32_t mh = m >> (16 * h);
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        if (((mh >> (4 * g)) & 0xfu) == 0) {
#pragma unroll
                            for (int i = 4 * g; i < 4 * g + 4; ++i) {
                                acc = add2_rn(acc, x[i]);
                            }
                        } else {
#pragma unroll
                            for (int i = 4 * g; i < 4 * g + 4; ++i) {
                                if (mh & (1u << i)) {
                                    start_run(rl);
                                }
                                acc = add2_rn(acc, x[i]);
                            }
                        }
                    }
                }
                s = (s + 1 == S) ? 0 : s + 1;
                if (s == 0) {
                    phase ^= 1u;
                }
                r = rbase + rl;
            }
            if constexpr (TM) {
                if (SEQ || bin != a.nbins) {
                    ptx::tmem_st2(T + 2 * bin, acc.x, acc.y);
                }
                ptx::tmem_wait_ld(nacc.x, nacc.y);
                ptx::tmem_wait_st();
            } else {
                A[bin * kWarp] = acc;
            }
            if (r != nr) {
                atomicOr(a.status, dev::kStatusBadTable);
            }
            return true;
        };
        bool ok;
        if (tm) {
            ok = a.seq[f] != 0 ? consume(std::true_type{}, std::true_type{})
                               : consume(std::false_type{}, std::true_type{});
        } else {
            ok = a.seq[f] != 0 ? consume(std::true_type{}, std::false_type{})
                               : consume(std::false_type{}, std::false_type{});
        }
        bool store;
        const uint32_t seg = lane_segment(a, seg0, lane, &store);
        float* out = a.fold + (static_cast<size_t>(seg) * a.nfreq + f) * 2 * a.nbins;
        if (ok && tm) {
            // every lane reads (warp-collective); lanes past nseg do not store
            for (uint32_t b = 0; b < a.nbins; b += 4) {
                float4 e4, v4;
                ptx::tmem_ld2(T + 2 * b, e4.x, v4.x);
                ptx::tmem_ld2(T + 2 * b + 2, e4.y, v4.y);
                ptx::tmem_ld2(T + 2 * b + 4, e4.z, v4.z);
                ptx::tmem_ld2(T + 2 * b + 6, e4.w, v4.w);
                ptx::tmem_wait_ld4(e4, v4);
                if (store) {
                    reinterpret_cast<float4*>(out)[b / 4] = e4;
                    reinterpret_cast<float4*>(out + a.nbins)[b / 4] = v4;
                }
            }
        } else if (ok && store) {
            for (uint32_t b = 0; b < a.nbins; b += 4) {
                const float2 p0 = A[b * kWarp], p1 = A[(b + 1) * kWarp];
                const float2 p2 = A[(b + 2) * kWarp], p3 = A[(b + 3) * kWarp];
                reinterpret_cast<float4*>(out)[b / 4] = make_float4(p0.x, p1.x, p2.x, p3.x);
                reinterpret_cast<float4*>(out + a.nbins)[b / 4] = make_float4(p0.y, p1.y, p2.y, p3.y);
            }
        }
    }
    ptx::tmem_fence_before_sync();
    __syncthreads();
    if (warp == W) {
        ptx::tmem_fence_after_sync();
        ptx::tmem_dealloc(tbase, kTmemCols);
    }
}

// Valid segments of series i, in whole groups of 8: the segments that hold
// any of its lens[i] samples, rounded up to 8 (at most nseg).
__device__ __forceinline__ uint32_t valid_segments8(uint64_t len, uint32_t nseg, uint64_t seglen) {
    const uint64_t used = (len + seglen - 1) / seglen;
    const uint64_t r8 = (used + 7) / 8 * 8;
    return static_cast<uint32_t>(r8 < nseg ? r8 : nseg);
}

// Group table of a batch (one block): tab[0] = number of groups, tab[1 ..
// nbatch] = each series' first group, tab[1 + nbatch ..] = each group's first
// row (series i's groups follow those of series < i).
__global__ void seg_groups_kernel(const uint64_t* __restrict__ lens, uint32_t nbatch, uint32_t nseg,
                                  uint64_t seglen, uint32_t* __restrict__ tab) {
    uint32_t* first = tab + 1;
    uint32_t* rows = tab + 1 + nbatch;
    if (threadIdx.x == 0) {
        uint32_t total = 0;
        for (uint32_t i = 0; i < nbatch; ++i) {
            first[i] = total;
            total += valid_segments8(lens[i], nseg, seglen) / 8;
        }
        tab[0] = total;
    }
    __syncthreads();
    for (uint32_t i = 0; i < nbatch; ++i) {
        const uint32_t n = valid_segments8(lens[i], nseg, seglen) / 8;
        for (uint32_t g = threadIdx.x; g < n; g += blockDim.x) {
            rows[first[i] + g] = i * nseg + 8 * g;
        }
    }
}

// Zeroes the fold of every segment that group mode skipped (all samples
// zero, so the fold is +0.0 in every bin, as folding them would give: a sum
// that starts at +0.0 stays +0.0 when +0.0 is added). Block = one segment.
__global__ void zero_skipped_kernel(const uint64_t* __restrict__ lens, uint32_t nseg, uint64_t seglen,
                                    uint64_t seg_floats, float* __restrict__ fold) {
    const uint32_t series = blockIdx.x / nseg;
    const uint32_t seg = blockIdx.x - series * nseg;
    if (seg < valid_segments8(lens[series], nseg, seglen)) {
        return;
    }
    float* out = fold + static_cast<uint64_t>(blockIdx.x) * seg_floats;
    if (seg_floats % 4 == 0) {
        float4* o4 = reinterpret_cast<float4*>(out);
        for (uint64_t i = threadIdx.x; i < seg_floats / 4; i += blockDim.x) {
            o4[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    } else {
        for (uint64_t i = threadIdx.x; i < seg_floats; i += blockDim.x) {
            out[i] = 0.0f;
        }
    }
}

// ev[i] = (e[i], v[i]) for i < n.
__global__ void interleave_kernel(const float* __restrict__ e, const float* __restrict__ v,
                                  float2* __restrict__ ev, uint64_t n, bool vec4) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (vec4) {
        const uint64_t n4 = n / 4;
        for (uint64_t i = t0; i < n4; i += stride) {
            const float4 a = __ldg(reinterpret_cast<const float4*>(e) + i);
            const float4 b = __ldg(reinterpret_cast<const float4*>(v) + i);
            float4* o = reinterpret_cast<float4*>(ev) + 2 * i;
            o[0] = make_float4(a.x, b.x, a.y, b.y);
            o[1] = make_float4(a.z, b.z, a.w, b.w);
        }
        for (uint64_t i = 4 * n4 + t0; i < n; i += stride) {
            ev[i] = make_float2(__ldg(e + i), __ldg(v + i));
        }
    } else {
        for (uint64_t i = t0; i < n; i += stride) {
            ev[i] = make_float2(__ldg(e + i), __ldg(v + i));
        }
    }
}

// 2-D map over one row of the series viewed as [nseg][seglen]; box 32
// samples x 32 segments, 128-byte swizzle; rows past nseg read as zero.
void encode_series_map(CUtensorMap* map, const float* base, uint64_t seglen, uint64_t nseg) {
    cuuint64_t dims[2] = {seglen, nseg};
    cuuint64_t strides[1] = {seglen * sizeof(float)};
    cuuint32_t box[2] = {32, 32};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = tensor_map_encoder()(
        map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box,
        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fail(LK_ERR_CUDA, "cuTensorMapEncodeTiled failed for the brute-fold input");
    }
}

// Interleaved series viewed as [nseg][2 * seglen] floats; box 32 floats
// (16 samples' pairs) x 32 segments, 128-byte swizzle; reads past a row's end
// or past nseg are zero.
void encode_ev_map(CUtensorMap* map, const float2* base, uint64_t seglen, uint64_t nseg,
                   uint32_t box_rows = 32) {
    cuuint64_t dims[2] = {2 * seglen, nseg};
    cuuint64_t strides[1] = {2 * seglen * sizeof(float)};
    cuuint32_t box[2] = {32, box_rows};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = tensor_map_encoder()(
        map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float2*>(base), dims, strides, box,
        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fail(LK_ERR_CUDA, "cuTensorMapEncodeTiled failed for the brute-fold input");
    }
}

}  // namespace

// cuTensorMapEncodeTiled from the driver (no link-time dependency on libcuda).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        LK_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000,
                                                 cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || p == nullptr) {
            fail(LK_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

BruteFoldDevice::BruteFoldDevice(const std::vector<double>& freqs, uint64_t segment_len,
                                 uint64_t nbins, uint64_t nsamps, double tsamp, double t_ref,
                                 uint32_t* d_status)
    : m_nfreq(freqs.size()),
      m_seglen(segment_len),
      m_nbins(nbins),
      m_nsamps(nsamps),
      m_status(d_status) {
    require(!freqs.empty(), "BruteFold: Frequency array is empty");
    require(segment_len > 0 && nsamps % segment_len == 0,
            "BruteFold: Number of samples is not a multiple of segment length");
    require(nbins >= 1, "BruteFold: nbins must be positive");
    for (double f : freqs) {
        require(f >= 0.0, "Frequency must be positive");
    }
    require(segment_len % 4 == 0,
            "BruteFold: the segment length must be a multiple of 4 samples (TMA row stride)");
    require(segment_len <= 0x7fffffffULL && m_nfreq <= 0x7fffffffULL,
            "BruteFold: sizes exceed 31 bits");
    require(nbins <= 65535, "BruteFold: nbins must be below 65536");
    m_nseg = nsamps / segment_len;
    // Words past the segment end have no run starts; their samples are read
    // as zeros (TMA fill) and adding +0.0 leaves every sum unchanged (a sum
    // that starts at +0.0 is never -0.0 in round-to-nearest).
    m_nwords = (segment_len + 31) / 32;
    m_wide_bins = nbins > 256;

    // Consumer warps per block: as many (frequency, row) accumulators as fit
    // next to the ring, then trimmed so the grid fills whole waves of SMs.
    // Ring depth: consumers are not starved even at 2 words (a B200 sweep of
    // 2 .. 16 words on the 2^22-sample accelerated workload changed nothing
    // but the shared memory left for accumulators), so 3 words leave the
    // most for accumulator warps. LOKI_B200_BF_STAGES overrides it (2 .. 16).
    uint32_t stages = 3;
    if (const char* env = std::getenv("LOKI_B200_BF_STAGES")) {
        stages = std::max<uint32_t>(2, std::min<uint32_t>(kMaxStages, std::atoi(env)));
    }
    // Rows per warp: both when two rows' accumulators of nbins <= 64 leave
    // room for >= 11 warps per block, else one (LOKI_B200_BF_ROWS overrides).
    uint32_t rows = m_nbins <= 64 ? 2 : 1;
    if (const char* env = std::getenv("LOKI_B200_BF_ROWS")) {
        rows = std::atoi(env) == 1 ? 1 : 2;
    }
    uint32_t warps = 0;  // 0: the wave-count rule below
    if (const char* env = std::getenv("LOKI_B200_BF_WARPS")) {
        warps = static_cast<uint32_t>(std::max(1, std::atoi(env)));
    }
    require(configure(rows, warps, stages),
            "BruteFold: nbins too large for the shared-memory accumulators");

    // Run tables, one frequency per task (host threads; same arithmetic as
    // the reference's BruteFold::compute_phase_time_domain, lib/fold.cpp:113-142).
    std::vector<uint32_t> masks(m_nfreq * m_nwords, 0u);
    std::vector<std::vector<uint16_t>> per_f(m_nfreq);
    const unsigned nthreads =
        std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 32u));
    auto work = [&](unsigned tid) {
        for (uint64_t f = tid; f < m_nfreq; f += nthreads) {
            uint32_t* mw = masks.data() + f * m_nwords;
            auto& rb = per_f[f];
            uint32_t prev = 0xffffffffu;
            for (uint64_t i = 0; i < segment_len; ++i) {
                const double proper_time = (static_cast<double>(i) * tsamp) - t_ref;
                const uint32_t b = host_phase_bin(proper_time, freqs[f], nbins);
                if (b != prev) {
                    mw[i / 32] |= 1u << (i % 32);
                    rb.push_back(static_cast<uint16_t>(b));
                    prev = b;
                }
            }
        }
    };
    {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < nthreads; ++t) {
            pool.emplace_back(work, t);
        }
        for (auto& t : pool) {
            t.join();
        }
    }
    // Frequencies whose run bins step by one bin (mod nbins) at every run.
    std::vector<uint8_t> seq(m_nfreq, 0);
    for (uint64_t f = 0; f < m_nfreq; ++f) {
        const auto& rb = per_f[f];
        bool ok = !rb.empty();
        for (size_t k = 1; ok && k < rb.size(); ++k) {
            ok = rb[k] == (rb[k - 1] + 1) % nbins;
        }
        seq[f] = ok ? 1 : 0;
    }
    std::vector<uint64_t> off(m_nfreq), nruns(m_nfreq);
    uint64_t total = 0;
    for (uint64_t f = 0; f < m_nfreq; ++f) {
        off[f] = total;
        nruns[f] = per_f[f].size();
        total += per_f[f].size();
    }
    const size_t bsz = m_wide_bins ? 2 : 1;
    std::vector<unsigned char> bins(std::max<uint64_t>(total, 1) * bsz);
    for (uint64_t f = 0; f < m_nfreq; ++f) {
        for (uint64_t k = 0; k < per_f[f].size(); ++k) {
            if (m_wide_bins) {
                std::memcpy(bins.data() + (off[f] + k) * 2, &per_f[f][k], 2);
            } else {
                bins[off[f] + k] = static_cast<unsigned char>(per_f[f][k]);
            }
        }
    }
    m_masks.alloc(sizeof(uint32_t) * masks.size());
    LK_CUDA(cudaMemcpy(m_masks.ptr, masks.data(), m_masks.bytes, cudaMemcpyHostToDevice));
    m_bins.alloc(bins.size());
    LK_CUDA(cudaMemcpy(m_bins.ptr, bins.data(), bins.size(), cudaMemcpyHostToDevice));
    m_bin_off.alloc(sizeof(uint64_t) * m_nfreq);
    LK_CUDA(cudaMemcpy(m_bin_off.ptr, off.data(), m_bin_off.bytes, cudaMemcpyHostToDevice));
    m_nruns.alloc(sizeof(uint64_t) * m_nfreq);
    LK_CUDA(cudaMemcpy(m_nruns.ptr, nruns.data(), m_nruns.bytes, cudaMemcpyHostToDevice));
    m_seq.alloc(m_nfreq);
    LK_CUDA(cudaMemcpy(m_seq.ptr, seq.data(), m_nfreq, cudaMemcpyHostToDevice));
    m_nseq = static_cast<uint64_t>(std::count(seq.begin(), seq.end(), uint8_t{1}));
}

// Launch shape: rows (E, V) per consumer warp, consumer warps per block
// (0: the fewest waves of blocks over the SMs among W >= 3/4 of the most that
// fit, the larger W on a tie -- the kernel is latency-bound per warp, so
// block time hardly depends on W) and the depth of the shared-memory ring.
// Returns false (and changes nothing) when the shape does not fit.
uint32_t BruteFoldDevice::max_tmem_warps(uint32_t smem_warps) const {
    // packed form, nbins a multiple of 4 up to 256, 2 * nbins columns per
    // warp, four warps (one per TMEM lane quadrant) per column block, block
    // <= 24 consumer warps
    if (m_nbins > 256 || m_nbins % 4 != 0 || smem_warps + 1 >= static_cast<uint32_t>(kMaxWarpsTm)) {
        return 0;
    }
    const uint32_t blocks = kTmemCols / static_cast<uint32_t>(2 * m_nbins);
    return std::min<uint32_t>(4 * blocks, static_cast<uint32_t>(kMaxWarpsTm) - 1 - smem_warps);
}

bool BruteFoldDevice::configure(uint32_t rows, uint32_t warps, uint32_t stages, uint32_t tmem) {
    if ((rows != 1 && rows != 2) || stages < 2 || stages > kMaxStages) {
        return false;
    }
    const size_t ring = stages * kStageBytes + 2 * stages * sizeof(uint64_t);
    const size_t per_warp = rows * (m_nbins + 1) * kWarp * sizeof(float);
    if (tmem > 0) {
        // shared-memory warps = warps - tmem, each with its accumulators
        if (rows != 2 || warps <= tmem || tmem > max_tmem_warps(warps - tmem)) {
            return false;
        }
        const size_t smem = ring + 16 + static_cast<size_t>(warps - tmem) * per_warp;
        if (smem > kSmemLimit || (m_nfreq + warps - 1) / warps > 65535) {
            return false;
        }
        m_rows = rows;
        m_warps = warps;
        m_stages = stages;
        m_tmem = tmem;
        // at least half the SM's shared memory: one block per SM, so a
        // second block never waits for the first one's tensor memory
        m_smem = std::max<size_t>(smem, 116 * 1024);
        m_map_e_ptr = nullptr;
        m_map_ev_ptr = nullptr;
        return true;
    }
    if (ring + per_warp > kSmemLimit) {
        return false;
    }
    const uint32_t wmax = static_cast<uint32_t>(
        std::min<size_t>((kSmemLimit - ring) / per_warp, kMaxConsumers));
    const uint64_t nitems = (rows == 2 ? 1 : 2) * m_nfreq;
    uint32_t w = warps;
    if (w == 0) {
        int dev = 0, nsm = 148;
        LK_CUDA(cudaGetDevice(&dev));
        LK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const uint64_t xblocks = (m_nseg + kWarp - 1) / kWarp;
        uint64_t best = ~0ull;
        for (uint32_t c = std::max<uint32_t>(1, (3 * wmax + 3) / 4); c <= wmax; ++c) {
            const uint64_t blocks = xblocks * ((nitems + c - 1) / c);
            const uint64_t waves = (blocks + nsm - 1) / nsm;
            if (waves <= best) {
                best = waves;
                w = c;
            }
        }
    }
    if (w < 1 || w > wmax || (nitems + w - 1) / w > 65535) {
        return false;
    }
    m_rows = rows;
    m_warps = w;
    m_stages = stages;
    m_tmem = 0;
    m_smem = ring + w * per_warp;
    m_map_e_ptr = nullptr;  // the input binding depends on the rows
    m_map_ev_ptr = nullptr;
    return true;
}

uint32_t BruteFoldDevice::max_warps(uint32_t rows, uint32_t stages) const {
    const size_t ring = stages * kStageBytes + 2 * stages * sizeof(uint64_t);
    const size_t per_warp = rows * (m_nbins + 1) * kWarp * sizeof(float);
    if (ring + per_warp > kSmemLimit) {
        return 0;
    }
    return static_cast<uint32_t>(std::min<size_t>((kSmemLimit - ring) / per_warp, kMaxConsumers));
}

uint64_t BruteFoldDevice::device_bytes() const {
    return m_masks.bytes + m_bins.bytes + m_bin_off.bytes + m_nruns.bytes + m_stage.bytes +
           m_ev.bytes + m_seq.bytes + m_groups.bytes;
}

// The TMA maps read the series in place; a base address that is not 16-byte
// aligned (a TMA requirement) is first copied into an aligned staging buffer.
// A batch of nbatch series stored back to back is folded as one series of
// nbatch * nseg segments: every segment is folded from its own start.
void BruteFoldDevice::bind_inputs(const float* d_ts_e, const float* d_ts_v, cudaStream_t s,
                                  uint64_t nbatch) {
    require(nbatch >= 1, "BruteFold: nbatch must be positive");
    const uint64_t n = nbatch * m_nsamps;
    if (m_rows == 2) {
        if (m_ev.bytes < n * sizeof(float2)) {
            m_ev.alloc(n * sizeof(float2));
        }
        const bool vec4 = (reinterpret_cast<uintptr_t>(d_ts_e) % 16 == 0) &&
                          (reinterpret_cast<uintptr_t>(d_ts_v) % 16 == 0);
        int dev = 0, nsm = 148;
        LK_CUDA(cudaGetDevice(&dev));
        LK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const uint64_t want = (n / (vec4 ? 4 : 1) + 255) / 256;
        const auto blocks = static_cast<unsigned>(
            std::max<uint64_t>(1, std::min<uint64_t>(want, static_cast<uint64_t>(nsm) * 8)));
        interleave_kernel<<<blocks, 256, 0, s>>>(d_ts_e, d_ts_v, m_ev.as<float2>(), n, vec4);
        LK_CUDA(cudaGetLastError());
        if (m_ev.ptr != m_map_ev_ptr || nbatch != m_map_batch) {
            encode_ev_map(&m_tmap_ev, m_ev.as<float2>(), m_seglen, nbatch * m_nseg);
            encode_ev_map(&m_tmap_ev8, m_ev.as<float2>(), m_seglen, nbatch * m_nseg, 8);
            m_map_ev_ptr = m_ev.ptr;
            m_map_batch = nbatch;
        }
        m_map_e_ptr = d_ts_e;  // marks the inputs as bound
        return;
    }
    const float* e = d_ts_e;
    const float* v = d_ts_v;
    const bool aligned = (reinterpret_cast<uintptr_t>(e) % 16 == 0) &&
                         (reinterpret_cast<uintptr_t>(v) % 16 == 0);
    if (!aligned) {
        if (m_stage.bytes < 2 * n * sizeof(float)) {
            m_stage.alloc(2 * n * sizeof(float));
        }
        float* se = m_stage.as<float>();
        float* sv = se + n;
        LK_CUDA(cudaMemcpyAsync(se, e, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        LK_CUDA(cudaMemcpyAsync(sv, v, n * sizeof(float), cudaMemcpyDeviceToDevice, s));
        e = se;
        v = sv;
    }
    if (e != m_map_e_ptr || v != m_map_v_ptr || nbatch != m_map_batch) {
        encode_series_map(&m_tmap_e, e, m_seglen, nbatch * m_nseg);
        encode_series_map(&m_tmap_v, v, m_seglen, nbatch * m_nseg);
        m_map_e_ptr = e;
        m_map_v_ptr = v;
        m_map_batch = nbatch;
    }
}

void BruteFoldDevice::fold(float* d_fold, cudaStream_t s, const uint64_t* d_lens) {
    require(m_map_e_ptr != nullptr, "BruteFold: inputs not bound");
    FoldArgs a{};
    a.masks = m_masks.as<uint32_t>();
    a.bins = m_bins.ptr;
    a.bin_off = m_bin_off.as<uint64_t>();
    a.nruns = m_nruns.as<uint64_t>();
    a.seq = m_seq.as<uint8_t>();
    const uint64_t nseg = m_map_batch * m_nseg;  // segments of the bound batch
    require(nseg <= 0x7fffffffULL, "BruteFold: too many segments");
    a.nfreq = static_cast<uint32_t>(m_nfreq);
    a.nseg = static_cast<uint32_t>(nseg);
    a.nbins = static_cast<uint32_t>(m_nbins);
    a.nwords = static_cast<uint32_t>(m_nwords);
    a.warps = m_warps;
    a.smem_warps = m_warps - m_tmem;
    a.stages = m_stages;
    a.fold = d_fold;
    a.status = m_status;
    const uint64_t nitems = (m_rows == 2 ? 1 : 2) * m_nfreq;
    dim3 grid(static_cast<unsigned>((nseg + kWarp - 1) / kWarp),
              static_cast<unsigned>((nitems + m_warps - 1) / m_warps));
    // Group mode: only the segments that hold samples are folded (in groups
    // of 8); the grid keeps its full size so that a captured graph stays
    // valid for any lengths, and blocks past the groups return at once.
    const bool grouped = d_lens != nullptr && m_rows == 2 && m_nseg % 8 == 0;
    if (grouped) {
        const uint64_t ngmax = nseg / 8;
        const uint64_t words = 1 + m_map_batch + ngmax;
        if (m_groups.bytes < words * sizeof(uint32_t)) {
            m_groups.alloc(words * sizeof(uint32_t));
        }
        uint32_t* tab = m_groups.as<uint32_t>();
        seg_groups_kernel<<<1, 256, 0, s>>>(d_lens, static_cast<uint32_t>(m_map_batch),
                                            static_cast<uint32_t>(m_nseg), m_seglen, tab);
        LK_CUDA(cudaGetLastError());
        a.ngroups = tab;
        a.groups = tab + 1 + m_map_batch;
        grid.x = static_cast<unsigned>((ngmax + 3) / 4);
    }
    auto launch = [&](auto kern) {
        LK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(m_smem)));
        kern<<<grid, (m_warps + 1) * kWarp, m_smem, s>>>(m_tmap_e, m_tmap_v, a);
    };
    auto launch_pk = [&](auto kern) {
        LK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(m_smem)));
        kern<<<grid, (m_warps + 1) * kWarp, m_smem, s>>>(m_tmap_ev, m_tmap_ev8, a);
    };
    if (m_rows == 2 && m_tmem > 0) {
        LK_CUDA(cudaFuncSetAttribute(brute_fold_pk_tm_kernel<uint8_t>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(m_smem)));
        brute_fold_pk_tm_kernel<uint8_t>
            <<<grid, (m_warps + 1) * kWarp, m_smem, s>>>(m_tmap_ev, m_tmap_ev8, a);
    } else if (m_rows == 2) {
        m_wide_bins ? launch_pk(brute_fold_pk_kernel<uint16_t>)
                    : launch_pk(brute_fold_pk_kernel<uint8_t>);
    } else {
        m_wide_bins ? launch(brute_fold_mask_kernel<uint16_t, 1>)
                    : launch(brute_fold_mask_kernel<uint8_t, 1>);
    }
    LK_CUDA(cudaGetLastError());
    if (grouped) {
        zero_skipped_kernel<<<static_cast<unsigned>(nseg), 256, 0, s>>>(
            d_lens, static_cast<uint32_t>(m_nseg), m_seglen, m_nfreq * 2 * m_nbins, d_fold);
        LK_CUDA(cudaGetLastError());
    }
}

}  // namespace lk
