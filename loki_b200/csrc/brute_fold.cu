// Brute fold (level 0 of the FFA) on sm_100a.
//
// out[seg, f, r, b] = sum over samples i of segment seg whose phase bin at
// frequency f is b, of ts_r[seg * seglen + i], added in increasing i starting
// from 0.0f -- the reference's order (lib/fold.cpp:113-142,
// lib/kernels.cpp:550-580,1132-1154), so results are bit-identical.
//
// Plan-time tables (host, once per plan): the sample -> bin map of one
// segment is the same for every segment. For each frequency it is encoded as
// the sequence of runs of equal bin in sample order, split at chunk
// boundaries (C samples): entry = (bin << 16) | length, plus the number of
// entries in each chunk.
//
// Execution:
//  * the series is transposed into xT[r][i][seg'] (seg' padded to a multiple
//    of the segment tile SW = 32 * SPL), so the SW segments of one sample are
//    one contiguous row;
//  * a block owns one segment tile and W (frequency, row) pairs, one per
//    consumer warp; lane l holds segments l*SPL .. l*SPL + SPL-1 of the tile
//    (one vector load covers them). All lanes of a warp follow the same run
//    sequence, so control flow is uniform and its cost is shared by 32*SPL
//    segments;
//  * a producer thread streams chunks of C samples x SW segments x 2 rows into
//    a 3-stage shared-memory ring with TMA; each consumer replays its runs:
//    one accumulator vector load and store per run ([bin][lane] layout,
//    conflict-free), one vector sample load + SPL adds per sample;
//  * the entries of the next chunk are loaded (coalesced, one per lane) while
//    the current chunk is processed and broadcast with warp shuffles.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>

#include <cudaTypedefs.h>

#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_ptx.cuh"

namespace lk {

namespace {

constexpr int kWarp = 32;
constexpr int kStages = 3;
constexpr uint32_t kMaxChunk = 128;       // entries per chunk fit 4 registers per lane
constexpr uint32_t kStageRowFloats = 4096; // C * SW per row and stage (16 KiB)
constexpr size_t kSmemLimit = 227 * 1024;
constexpr int kMaxConsumers = 31;          // + 1 producer warp = 1024 threads

template <int SPL> struct Vec;
template <> struct Vec<1> {
    using T = float;
    __device__ static void add(T& a, const T& x) { a = __fadd_rn(a, x); }
    __device__ static T zero() { return 0.0f; }
    __device__ static float get(const T& v, int) { return v; }
};
template <> struct Vec<2> {
    using T = float2;
    __device__ static void add(T& a, const T& x) {
        a.x = __fadd_rn(a.x, x.x);
        a.y = __fadd_rn(a.y, x.y);
    }
    __device__ static T zero() { return make_float2(0.0f, 0.0f); }
    __device__ static float get(const T& v, int k) { return k == 0 ? v.x : v.y; }
};
template <> struct Vec<4> {
    using T = float4;
    __device__ static void add(T& a, const T& x) {
        a.x = __fadd_rn(a.x, x.x);
        a.y = __fadd_rn(a.y, x.y);
        a.z = __fadd_rn(a.z, x.z);
        a.w = __fadd_rn(a.w, x.w);
    }
    __device__ static T zero() { return make_float4(0.0f, 0.0f, 0.0f, 0.0f); }
    __device__ static float get(const T& v, int k) {
        return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
    }
};

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

// ---- input transpose ------------------------------------------------------

// ts_r[seg * seglen + i] -> xT[r][i][seg]; 32x32 tiles through shared memory.
__global__ void transpose_kernel(const float* __restrict__ ts_e, const float* __restrict__ ts_v,
                                 float* __restrict__ xT, uint32_t seglen, uint32_t nseg,
                                 uint32_t nseg_pad) {
    __shared__ float tile[32][33];
    const uint32_t r = blockIdx.z;
    const float* src = r == 0 ? ts_e : ts_v;
    const uint32_t i0 = blockIdx.x * 32;  // sample
    const uint32_t s0 = blockIdx.y * 32;  // segment
    const uint32_t tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (uint32_t k = ty; k < 32; k += 8) {
        const uint32_t s = s0 + k, i = i0 + tx;
        tile[k][tx] = (s < nseg && i < seglen) ? __ldg(src + static_cast<uint64_t>(s) * seglen + i)
                                               : 0.0f;
    }
    __syncthreads();
    float* dst = xT + static_cast<uint64_t>(r) * seglen * nseg_pad;
    for (uint32_t k = ty; k < 32; k += 8) {
        const uint32_t i = i0 + k, s = s0 + tx;
        if (i < seglen && s < nseg_pad) {
            dst[static_cast<uint64_t>(i) * nseg_pad + s] = tile[tx][k];
        }
    }
}

// ---- the fold ---------------------------------------------------------------

struct FoldArgs {
    const uint32_t* entries;   // all frequencies
    const uint64_t* offsets;   // first entry of each frequency
    const uint8_t* counts;     // [nfreq][nchunks] entries per chunk
    uint32_t nfreq;
    uint32_t nseg;
    uint32_t nbins;
    uint32_t chunk;            // C <= kMaxChunk
    uint32_t nchunks;
    uint32_t warps;            // W consumer warps per block
    float* fold;
    uint32_t* status;
};

// Loads the entries of one chunk: lane j holds entries j, j+32, j+64, j+96.
__device__ __forceinline__ void load_chunk_entries(const uint32_t* e, uint32_t n, int lane,
                                                   uint32_t (&r)[4]) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const uint32_t k = static_cast<uint32_t>(lane + 32 * j);
        r[j] = k < n ? __ldg(e + k) : 0u;
    }
}

template <int SPL, int R>
__global__ void __launch_bounds__(1024, 1)
    brute_fold_runs_kernel(const __grid_constant__ CUtensorMap tmap, FoldArgs a) {
    using V = typename Vec<SPL>::T;
    constexpr uint32_t SW = kWarp * SPL;  // segments per tile
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t C = a.chunk;
    const uint32_t stage_floats = 2 * C * SW;
    float* xs = reinterpret_cast<float*>(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + kStages * stage_floats * sizeof(float));
    uint64_t* empty = full + kStages;
    V* accs = reinterpret_cast<V*>(empty + kStages);

    const int warp = threadIdx.x / kWarp;
    const int lane = threadIdx.x % kWarp;
    const int W = static_cast<int>(a.warps);
    // Work items: (frequency, row) pairs when R == 1, frequencies when R == 2.
    const uint32_t q0 = blockIdx.y * a.warps;  // first work item of the block
    const uint32_t nitems = (R == 1 ? 2 : 1) * a.nfreq;
    const int nconsumers = static_cast<int>(min(a.warps, nitems - q0));

    if (threadIdx.x == 0) {
        ptx::prefetch_tensormap(&tmap);
        for (int s = 0; s < kStages; ++s) {
            ptx::mbar_init(&full[s], 1);
            ptx::mbar_init(&empty[s], nconsumers * kWarp);
        }
        ptx::fence_barrier_init();
    }
    __syncthreads();

    if (warp == W) {
        // Producer: one thread issues every chunk's TMA load.
        if (lane == 0) {
            uint32_t issued = 0;
            for (uint32_t k = 0; k < a.nchunks; ++k) {
                const int s = static_cast<int>(k % kStages);
                if (k >= static_cast<uint32_t>(kStages) &&
                    !ptx::mbar_wait_bounded(&empty[s], ((k / kStages) - 1) & 1u, a.status,
                                            dev::kStatusWaitTimeout | dev::kStatusEmpty)) {
                    break;
                }
                ptx::mbar_arrive_expect_tx(&full[s], stage_floats * sizeof(float));
                ptx::tma_load_3d(xs + static_cast<size_t>(s) * stage_floats, &tmap, &full[s],
                                 static_cast<int>(blockIdx.x * SW), static_cast<int>(k * C), 0);
                ++issued;
            }
            // Stay resident until the last loads have landed (bounded).
            const uint32_t first = issued > static_cast<uint32_t>(kStages) ? issued - kStages : 0;
            for (uint32_t k = first; k < issued; ++k) {
                ptx::mbar_wait_bounded(&full[k % kStages], (k / kStages) & 1u, a.status,
                                       dev::kStatusWaitTimeout | dev::kStatusDrain);
            }
        }
        return;
    }
    if (warp >= nconsumers) {
        return;
    }

    const uint32_t q = q0 + static_cast<uint32_t>(warp);
    const uint32_t f = R == 1 ? (q >> 1) : q;
    const int row0 = R == 1 ? static_cast<int>(q & 1u) : 0;
    // Accumulators of this warp: [R rows][nbins][32 lanes] vectors; A[r][b * 32].
    V* A0 = accs + static_cast<size_t>(warp) * R * a.nbins * kWarp + lane;
    V* A1 = A0 + (R == 2 ? a.nbins * kWarp : 0);
    for (uint32_t b = 0; b < R * a.nbins; ++b) {
        A0[b * kWarp] = Vec<SPL>::zero();
    }
    const uint32_t* E = a.entries + a.offsets[f];
    const uint8_t* CNT = a.counts + static_cast<size_t>(f) * a.nchunks;

    uint32_t ne = CNT[0];
    uint32_t cur[4];
    load_chunk_entries(E, ne, lane, cur);
    uint32_t pos = ne;
    uint32_t phase = 0;
    int s = 0;
    for (uint32_t k = 0; k < a.nchunks; ++k) {
        // Prefetch the next chunk's entries while this one is processed.
        uint32_t ne_next = 0;
        uint32_t nxt[4] = {0u, 0u, 0u, 0u};
        if (k + 1 < a.nchunks) {
            ne_next = CNT[k + 1];
            load_chunk_entries(E + pos, ne_next, lane, nxt);
        }
        if (!ptx::mbar_wait_bounded(&full[s], phase, a.status,
                                    dev::kStatusWaitTimeout |
                                        (k == 0 ? dev::kStatusFirstFull : dev::kStatusFull))) {
            return;
        }
        // Row `row0` of stage s: [C samples][SW segments]; lane's vector column.
        // With R == 2 the V row follows at + C * SW floats.
        const V* xb = reinterpret_cast<const V*>(xs + static_cast<size_t>(s) * stage_floats +
                                                 static_cast<size_t>(row0) * C * SW) +
                      lane;
        const uint32_t vrow = C * kWarp;  // V-row offset in vectors
        uint32_t i = 0;
        for (uint32_t e = 0; e < ne; ++e) {
            const uint32_t src = e < 32 ? cur[0] : (e < 64 ? cur[1] : (e < 96 ? cur[2] : cur[3]));
            const uint32_t word = __shfl_sync(0xffffffffu, src, static_cast<int>(e & 31u));
            const uint32_t b = word >> 16;
            const uint32_t n = word & 0xffffu;
            V acc = A0[b * kWarp];
            V acc1 = R == 2 ? A1[b * kWarp] : Vec<SPL>::zero();
            const V* xp = xb + i * kWarp;
            uint32_t t = 0;
            for (; t + 4 <= n; t += 4) {
                const V x0 = xp[(t + 0) * kWarp];
                const V x1 = xp[(t + 1) * kWarp];
                const V x2 = xp[(t + 2) * kWarp];
                const V x3 = xp[(t + 3) * kWarp];
                if (R == 2) {
                    const V y0 = xp[vrow + (t + 0) * kWarp];
                    const V y1 = xp[vrow + (t + 1) * kWarp];
                    const V y2 = xp[vrow + (t + 2) * kWarp];
                    const V y3 = xp[vrow + (t + 3) * kWarp];
                    Vec<SPL>::add(acc1, y0);
                    Vec<SPL>::add(acc1, y1);
                    Vec<SPL>::add(acc1, y2);
                    Vec<SPL>::add(acc1, y3);
                }
                Vec<SPL>::add(acc, x0);
                Vec<SPL>::add(acc, x1);
                Vec<SPL>::add(acc, x2);
                Vec<SPL>::add(acc, x3);
            }
            for (; t < n; ++t) {
                Vec<SPL>::add(acc, xp[t * kWarp]);
                if (R == 2) {
                    Vec<SPL>::add(acc1, xp[vrow + t * kWarp]);
                }
            }
            A0[b * kWarp] = acc;
            if (R == 2) {
                A1[b * kWarp] = acc1;
            }
            i += n;
        }
        // Release the stage: every lane arrives (release semantics order its
        // reads before the producer's next TMA write into the stage).
        ptx::mbar_arrive(&empty[s]);
        s = (s + 1 == kStages) ? 0 : s + 1;
        if (s == 0) {
            phase ^= 1u;
        }
        pos += ne_next;
        ne = ne_next;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            cur[j] = nxt[j];
        }
    }

#pragma unroll
    for (int r = 0; r < R; ++r) {
        const V* A = r == 0 ? A0 : A1;
        const int row = row0 + r;
#pragma unroll
        for (int k = 0; k < SPL; ++k) {
            const uint32_t seg = blockIdx.x * SW + static_cast<uint32_t>(lane) * SPL + k;
            if (seg < a.nseg) {
                float* out =
                    a.fold + ((static_cast<size_t>(seg) * a.nfreq + f) * 2 + row) * a.nbins;
                if ((a.nbins & 3u) == 0) {
                    for (uint32_t b = 0; b < a.nbins; b += 4) {
                        reinterpret_cast<float4*>(out)[b / 4] =
                            make_float4(Vec<SPL>::get(A[b * kWarp], k),
                                        Vec<SPL>::get(A[(b + 1) * kWarp], k),
                                        Vec<SPL>::get(A[(b + 2) * kWarp], k),
                                        Vec<SPL>::get(A[(b + 3) * kWarp], k));
                    }
                } else {
                    for (uint32_t b = 0; b < a.nbins; ++b) {
                        out[b] = Vec<SPL>::get(A[b * kWarp], k);
                    }
                }
            }
        }
    }
}

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

// Segments per lane. One segment per lane measured fastest on B200 for the
// 2^22-sample, 256-segment, 64-bin accelerated workload (3.96 ms against 4.04
// for two and 4.85 for four): more segments per lane lengthen each run's
// shared-memory read-modify-write without saving decode work.
// LOKI_B200_BF_SPL (1, 2 or 4) overrides it for tuning.
uint32_t choose_spl(uint64_t /*nseg*/) {
    if (const char* env = std::getenv("LOKI_B200_BF_SPL")) {
        const int v = std::atoi(env);
        if (v == 1 || v == 2 || v == 4) {
            return static_cast<uint32_t>(v);
        }
    }
    return 1;
}

}  // namespace

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
    require(segment_len <= 0x7fffffffULL && m_nfreq <= 0x7fffffffULL,
            "BruteFold: sizes exceed 31 bits");
    m_nseg = nsamps / segment_len;
    m_spl = choose_spl(m_nseg);
    const uint64_t sw = kWarp * m_spl;
    m_nseg_pad = (m_nseg + sw - 1) / sw * sw;
    // Chunk: the largest power of two dividing segment_len, with C * SW per
    // row and stage at most kStageRowFloats.
    const uint64_t cmax = std::min<uint64_t>(kMaxChunk, kStageRowFloats / sw);
    m_chunk = 1;
    while (m_chunk < cmax && segment_len % (m_chunk * 2) == 0) {
        m_chunk *= 2;
    }
    m_nchunks = segment_len / m_chunk;
    // Consumer warps per block: as many (frequency, row) accumulators as fit
    // next to the stage ring.
    const size_t stages = kStages * 2 * m_chunk * sw * sizeof(float) + 2 * kStages * sizeof(uint64_t);
    // Rows per warp: one (E and V of a frequency on two warps of one block,
    // 3.96 ms against 4.15 ms for both rows on one warp on the workload
    // above), or two when LOKI_B200_BF_ROWS=2 asks and the accumulators fit.
    m_rows = 1;
    if (const char* env = std::getenv("LOKI_B200_BF_ROWS")) {
        m_rows = std::atoi(env) == 2 ? 2 : 1;
    }
    if (stages + 2 * static_cast<size_t>(m_nbins) * sw * sizeof(float) > kSmemLimit) {
        m_rows = 1;
    }
    const size_t per_warp = m_rows * static_cast<size_t>(m_nbins) * sw * sizeof(float);
    require(stages + per_warp <= kSmemLimit,
            "BruteFold: nbins too large for the shared-memory accumulators");
    m_warps = static_cast<uint32_t>(
        std::min<size_t>((kSmemLimit - stages) / per_warp, kMaxConsumers));
    if (m_rows == 1 && m_warps > 1) {
        m_warps &= ~1u;  // keep both rows of a frequency in one block
    }
    m_smem = stages + m_warps * per_warp;
    const uint64_t nitems = (m_rows == 1 ? 2 : 1) * m_nfreq;
    require((nitems + m_warps - 1) / m_warps <= 65535, "BruteFold: too many frequencies");

    // Run tables, one frequency per task (host threads; same arithmetic as
    // the reference's BruteFold::compute_phase_time_domain, lib/fold.cpp:113-142).
    std::vector<std::vector<uint32_t>> per_f(m_nfreq);
    std::vector<uint8_t> counts(m_nfreq * m_nchunks);
    const unsigned nthreads =
        std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 32u));
    auto work = [&](unsigned tid) {
        std::vector<uint32_t> bins(segment_len);
        for (uint64_t f = tid; f < m_nfreq; f += nthreads) {
            for (uint64_t i = 0; i < segment_len; ++i) {
                const double proper_time = (static_cast<double>(i) * tsamp) - t_ref;
                bins[i] = host_phase_bin(proper_time, freqs[f], nbins);
            }
            auto& ent = per_f[f];
            for (uint64_t k = 0; k < m_nchunks; ++k) {
                const uint64_t i0 = k * m_chunk, i1 = i0 + m_chunk;
                uint32_t n = 0;
                uint64_t i = i0;
                while (i < i1) {
                    uint64_t j = i + 1;
                    while (j < i1 && bins[j] == bins[i]) {
                        ++j;
                    }
                    ent.push_back((bins[i] << 16) | static_cast<uint32_t>(j - i));
                    ++n;
                    i = j;
                }
                counts[f * m_nchunks + k] = static_cast<uint8_t>(n);
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
    std::vector<uint64_t> off(m_nfreq);
    uint64_t total = 0;
    for (uint64_t f = 0; f < m_nfreq; ++f) {
        off[f] = total;
        total += per_f[f].size();
    }
    std::vector<uint32_t> entries;
    entries.reserve(total);
    for (auto& v : per_f) {
        entries.insert(entries.end(), v.begin(), v.end());
    }
    m_entries.alloc(sizeof(uint32_t) * std::max<uint64_t>(total, 1));
    LK_CUDA(cudaMemcpy(m_entries.ptr, entries.data(), sizeof(uint32_t) * total,
                       cudaMemcpyHostToDevice));
    m_offsets.alloc(sizeof(uint64_t) * m_nfreq);
    LK_CUDA(cudaMemcpy(m_offsets.ptr, off.data(), sizeof(uint64_t) * m_nfreq,
                       cudaMemcpyHostToDevice));
    m_counts.alloc(counts.size());
    LK_CUDA(cudaMemcpy(m_counts.ptr, counts.data(), counts.size(), cudaMemcpyHostToDevice));

    // Transposed input scratch and its TMA descriptor (box: SW segments x C
    // samples x 2 rows).
    m_xT.alloc(sizeof(float) * 2 * m_seglen * m_nseg_pad);
    LK_CUDA(cudaMemset(m_xT.ptr, 0, m_xT.bytes));
    cuuint64_t dims[3] = {m_nseg_pad, m_seglen, 2};
    cuuint64_t strides[2] = {m_nseg_pad * sizeof(float), m_seglen * m_nseg_pad * sizeof(float)};
    cuuint32_t box[3] = {static_cast<cuuint32_t>(sw), static_cast<cuuint32_t>(m_chunk), 2};
    cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = tensor_map_encoder()(
        &m_tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, m_xT.ptr, dims, strides, box, estr,
        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fail(LK_ERR_CUDA, "cuTensorMapEncodeTiled failed for the brute-fold input");
    }
}

uint64_t BruteFoldDevice::device_bytes() const {
    return m_entries.bytes + m_offsets.bytes + m_counts.bytes + m_xT.bytes;
}

void BruteFoldDevice::transpose(const float* d_ts_e, const float* d_ts_v, cudaStream_t s) {
    const auto seglen = static_cast<uint32_t>(m_seglen);
    const auto nseg = static_cast<uint32_t>(m_nseg);
    const auto nseg_pad = static_cast<uint32_t>(m_nseg_pad);
    dim3 tgrid((seglen + 31) / 32, nseg_pad / 32, 2);
    transpose_kernel<<<tgrid, dim3(32, 8), 0, s>>>(d_ts_e, d_ts_v, m_xT.as<float>(), seglen, nseg,
                                                   nseg_pad);
    LK_CUDA(cudaGetLastError());
}

void BruteFoldDevice::fold(float* d_fold, cudaStream_t s) {
    FoldArgs a{};
    a.entries = m_entries.as<uint32_t>();
    a.offsets = m_offsets.as<uint64_t>();
    a.counts = m_counts.as<uint8_t>();
    a.nfreq = static_cast<uint32_t>(m_nfreq);
    a.nseg = static_cast<uint32_t>(m_nseg);
    a.nbins = static_cast<uint32_t>(m_nbins);
    a.chunk = static_cast<uint32_t>(m_chunk);
    a.nchunks = static_cast<uint32_t>(m_nchunks);
    a.warps = m_warps;
    a.fold = d_fold;
    a.status = m_status;
    const uint64_t nitems = (m_rows == 1 ? 2 : 1) * m_nfreq;
    dim3 grid(static_cast<unsigned>(m_nseg_pad / (kWarp * m_spl)),
              static_cast<unsigned>((nitems + m_warps - 1) / m_warps));
    auto launch = [&](auto kern) {
        LK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(m_smem)));
        kern<<<grid, (m_warps + 1) * kWarp, m_smem, s>>>(m_tmap, a);
    };
    const int variant = static_cast<int>(m_spl) * 10 + static_cast<int>(m_rows);
    switch (variant) {
    case 42: launch(brute_fold_runs_kernel<4, 2>); break;
    case 41: launch(brute_fold_runs_kernel<4, 1>); break;
    case 22: launch(brute_fold_runs_kernel<2, 2>); break;
    case 21: launch(brute_fold_runs_kernel<2, 1>); break;
    case 12: launch(brute_fold_runs_kernel<1, 2>); break;
    default: launch(brute_fold_runs_kernel<1, 1>); break;
    }
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
