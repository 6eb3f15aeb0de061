// Brute fold (level 0 of the FFA) on sm_100a.
//
// out[seg, f, r, b] = sum over samples i of segment seg whose phase bin at
// frequency f is b, of ts_r[seg * seglen + i], summed in increasing i from
// 0.0f -- the reference's order (lib/fold.cpp:113-142,
// lib/kernels.cpp:550-580,1132-1154).
//
// Layout and work split:
//  * the series is transposed once per call into xT[r][i][seg'] (seg' padded
//    to a multiple of 32) so that 32 consecutive segments of one sample are
//    one 128-byte row;
//  * a warp owns 32 segments (one per lane) x one frequency x one row (E or
//    V). All lanes share the frequency's run table, so control flow is
//    uniform and the nbins accumulators live in registers (static indices
//    through a fully unrolled bin loop);
//  * a producer warp streams chunks of C samples x 32 segments x 2 rows into
//    an S-stage shared-memory ring with TMA; consumer warps read them with
//    conflict-free 4-byte loads (lane = segment = bank).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>

#include <cudaTypedefs.h>

#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_ptx.cuh"

namespace lk::bf {
// Defined in brute_fold_tma.cuh, instantiated in brute_fold_nb*.cu.
template <int NBINS>
void launch_tma(const CUtensorMap& tmap, const uint16_t* lens, const uint64_t* off,
                const uint32_t* nper, uint32_t nfreq, uint32_t nseg, uint32_t nseg_pad,
                uint32_t seglen, float* fold, uint32_t* status, cudaStream_t s);
constexpr int kChunk = 128;
}  // namespace lk::bf

namespace lk {

namespace {

constexpr int kWarp = 32;

// ---- plan-time run tables -------------------------------------------------

// Warp per frequency. Lanes compute the phase bins of 32 consecutive samples,
// the warp derives the virtual-bin index of each sample (cyclic forward
// distance from the previous sample's bin, inclusive scan), and either
// reports the number of virtual periods (fill == false) or accumulates the
// run lengths (fill == true).
__global__ void run_table_kernel(const double* __restrict__ freqs, uint32_t nfreq,
                                 uint32_t seglen, uint32_t nbins, double tsamp, double t_ref,
                                 bool fill, uint32_t* __restrict__ nper,
                                 const uint64_t* __restrict__ lens_off,
                                 uint16_t* __restrict__ lens, uint32_t* status) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) / kWarp;
    const uint32_t lane = threadIdx.x % kWarp;
    if (warp >= nfreq) {
        return;
    }
    const double freq = freqs[warp];
    uint16_t* L = fill ? lens + lens_off[warp] : nullptr;
    uint32_t prev_bin = 0;  // bin of the last sample of the previous chunk
    uint64_t v_base = 0;    // virtual index of that sample
    for (uint32_t i0 = 0; i0 < seglen; i0 += kWarp) {
        const uint32_t i = i0 + lane;
        const bool valid = i < seglen;
        uint32_t b = 0;
        if (valid) {
            const double proper_time = dev::dsub(dev::dmul(dev::u2d(i), tsamp), t_ref);
            b = dev::phase_idx_uint(proper_time, freq, nbins, 0.0);
        }
        uint32_t bprev = __shfl_up_sync(0xffffffffu, b, 1);
        if (lane == 0) {
            bprev = prev_bin;
        }
        uint64_t delta;
        if (i == 0) {
            delta = b;  // the first sample sits at virtual index = its bin
        } else {
            delta = valid ? static_cast<uint64_t>((b + nbins - bprev) % nbins) : 0;
        }
        // Inclusive scan of delta over the warp.
        uint64_t v = delta;
#pragma unroll
        for (int o = 1; o < kWarp; o <<= 1) {
            const uint64_t t = __shfl_up_sync(0xffffffffu, v, o);
            if (static_cast<int>(lane) >= o) {
                v += t;
            }
        }
        v += v_base;
        if (fill) {
            // One writer per distinct virtual index in this chunk: the last
            // lane of each run adds the run's length within the chunk.
            // Every lane executes both shuffles (full mask) before any
            // lane-dependent condition.
            const uint64_t vnext = __shfl_down_sync(0xffffffffu, v, 1);
            const uint64_t vprev = __shfl_up_sync(0xffffffffu, v, 1);
            const bool start = (lane == 0) || (v != vprev);
            const uint32_t starts = __ballot_sync(0xffffffffu, start && valid);
            const bool end = valid && ((lane == kWarp - 1) || (i + 1 >= seglen) || vnext != v);
            if (end) {
                const uint32_t upto = starts & (0xffffffffu >> (kWarp - 1 - lane));
                const uint32_t first = kWarp - 1 - __clz(upto);
                const uint32_t cnt = lane - first + 1;
                const uint32_t total = static_cast<uint32_t>(L[v]) + cnt;
                if (total > 0xffffu) {
                    atomicOr(status, dev::kStatusRunTooLong);
                }
                L[v] = static_cast<uint16_t>(total);
            }
        }
        const uint32_t last_lane = (seglen - i0 >= kWarp) ? kWarp - 1 : (seglen - i0 - 1);
        prev_bin = __shfl_sync(0xffffffffu, b, last_lane);
        v_base = __shfl_sync(0xffffffffu, v, last_lane);
    }
    if (!fill && lane == 0) {
        nper[warp] = static_cast<uint32_t>(v_base / nbins + 1);
    }
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

// Any nbins: same run replay, accumulators in shared memory ([bin][lane]
// per warp, conflict-free), samples read straight from the transposed
// global copy (coalesced 128-byte rows).
__global__ void brute_fold_generic_kernel(const float* __restrict__ xT,
                                          const uint16_t* __restrict__ lens,
                                          const uint64_t* __restrict__ lens_off,
                                          const uint32_t* __restrict__ nper, uint32_t nfreq,
                                          uint32_t nseg, uint32_t nseg_pad, uint32_t seglen,
                                          uint32_t nbins, float* __restrict__ fold) {
    extern __shared__ float accs[];  // [2 warps][nbins][32]
    const int warp = threadIdx.x / kWarp;  // row
    const int lane = threadIdx.x % kWarp;
    const uint32_t f = blockIdx.y;
    if (f >= nfreq) {
        return;
    }
    float* A = accs + static_cast<size_t>(warp) * nbins * kWarp;
    for (uint32_t b = 0; b < nbins; ++b) {
        A[b * kWarp + lane] = 0.0f;
    }
    const uint16_t* L = lens + lens_off[f];
    const uint64_t nv = static_cast<uint64_t>(nper[f]) * nbins;
    const float* x = xT + static_cast<size_t>(warp) * seglen * nseg_pad + blockIdx.x * kWarp + lane;
    uint32_t i = 0;
    for (uint64_t v = 0; v < nv; ++v) {
        const uint32_t n = L[v];
        if (n == 0) {
            continue;
        }
        const uint32_t b = static_cast<uint32_t>(v % nbins);
        float a = A[b * kWarp + lane];
        for (uint32_t t = 0; t < n; ++t, ++i) {
            a = __fadd_rn(a, __ldg(x + static_cast<size_t>(i) * nseg_pad));
        }
        A[b * kWarp + lane] = a;
    }
    const uint32_t seg = blockIdx.x * kWarp + lane;
    if (seg < nseg) {
        float* out = fold + ((static_cast<size_t>(seg) * nfreq + f) * 2 + warp) * nbins;
        for (uint32_t b = 0; b < nbins; ++b) {
            out[b] = A[b * kWarp + lane];
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

// Kernel shapes per nbins: chunk C samples, S pipeline stages, G frequencies
// (2G consumer warps) per block. Register budget: NBINS accumulators per
// thread, one block per SM.
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
    m_nseg_pad = (m_nseg + kWarp - 1) / kWarp * kWarp;

    // Run tables: pass 1 counts virtual periods, pass 2 fills run lengths.
    DeviceBuffer d_freqs(sizeof(double) * m_nfreq);
    LK_CUDA(cudaMemcpy(d_freqs.ptr, freqs.data(), sizeof(double) * m_nfreq,
                       cudaMemcpyHostToDevice));
    m_nper.alloc(sizeof(uint32_t) * m_nfreq);
    const unsigned threads = 256;
    const unsigned blocks = static_cast<unsigned>((m_nfreq * kWarp + threads - 1) / threads);
    run_table_kernel<<<blocks, threads>>>(d_freqs.as<double>(), static_cast<uint32_t>(m_nfreq),
                                          static_cast<uint32_t>(m_seglen),
                                          static_cast<uint32_t>(m_nbins), tsamp, t_ref, false,
                                          m_nper.as<uint32_t>(), nullptr, nullptr, m_status);
    LK_CUDA(cudaGetLastError());
    std::vector<uint32_t> nper(m_nfreq);
    LK_CUDA(cudaMemcpy(nper.data(), m_nper.ptr, sizeof(uint32_t) * m_nfreq,
                       cudaMemcpyDeviceToHost));
    std::vector<uint64_t> off(m_nfreq);
    uint64_t total = 0;
    for (uint64_t f = 0; f < m_nfreq; ++f) {
        off[f] = total;
        total += static_cast<uint64_t>(nper[f]) * m_nbins;
        // uint4 loads of run lengths need 16-byte aligned per-frequency tables.
        total = (total + 7) / 8 * 8;
    }
    m_lens_off.alloc(sizeof(uint64_t) * m_nfreq);
    LK_CUDA(cudaMemcpy(m_lens_off.ptr, off.data(), sizeof(uint64_t) * m_nfreq,
                       cudaMemcpyHostToDevice));
    m_lens.alloc(sizeof(uint16_t) * std::max<uint64_t>(total, 8));
    LK_CUDA(cudaMemset(m_lens.ptr, 0, m_lens.bytes));
    run_table_kernel<<<blocks, threads>>>(d_freqs.as<double>(), static_cast<uint32_t>(m_nfreq),
                                          static_cast<uint32_t>(m_seglen),
                                          static_cast<uint32_t>(m_nbins), tsamp, t_ref, true,
                                          m_nper.as<uint32_t>(), m_lens_off.as<uint64_t>(),
                                          m_lens.as<uint16_t>(), m_status);
    LK_CUDA(cudaGetLastError());
    LK_CUDA(cudaDeviceSynchronize());
    uint32_t st = 0;
    LK_CUDA(cudaMemcpy(&st, m_status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if ((st & dev::kStatusRunTooLong) != 0) {
        fail(LK_ERR_UNSUPPORTED, "BruteFold: a phase-bin run exceeds 65535 samples");
    }

    // Transposed input scratch and its TMA descriptor.
    m_xT.alloc(sizeof(float) * 2 * m_seglen * m_nseg_pad);
    LK_CUDA(cudaMemset(m_xT.ptr, 0, m_xT.bytes));
    const bool pow2_bins = m_nbins == 8 || m_nbins == 16 || m_nbins == 32 || m_nbins == 64 ||
                           m_nbins == 128;
    // LOKI_B200_BRUTE_FOLD=generic selects the shared-memory-accumulator
    // kernel for every nbins (same results; used to cross-check the
    // pipelined kernel).
    const char* force = std::getenv("LOKI_B200_BRUTE_FOLD");
    const bool force_generic = force != nullptr && std::string(force) == "generic";
    m_use_tma = !force_generic && pow2_bins && (m_seglen % bf::kChunk == 0);
    require(!m_use_tma || (m_nfreq + 3) / 4 <= 65535, "BruteFold: too many frequencies");
    if (m_use_tma) {
        cuuint64_t dims[3] = {m_nseg_pad, m_seglen, 2};
        cuuint64_t strides[2] = {m_nseg_pad * sizeof(float), m_seglen * m_nseg_pad * sizeof(float)};
        cuuint32_t box[3] = {static_cast<cuuint32_t>(kWarp), static_cast<cuuint32_t>(bf::kChunk), 2};
        cuuint32_t estr[3] = {1, 1, 1};
        const CUresult r = tensor_map_encoder()(
            &m_tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, m_xT.ptr, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            fail(LK_ERR_CUDA, "cuTensorMapEncodeTiled failed for the brute-fold input");
        }
    } else {
        const size_t smem = 2ull * m_nbins * kWarp * sizeof(float);
        require(smem <= 200 * 1024, "BruteFold: nbins too large for the generic kernel");
        require(m_nfreq <= 65535, "BruteFold: too many frequencies for the generic kernel");
        if (smem > 48 * 1024) {
            LK_CUDA(cudaFuncSetAttribute(brute_fold_generic_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)));
        }
    }
}

uint64_t BruteFoldDevice::device_bytes() const {
    return m_lens.bytes + m_lens_off.bytes + m_nper.bytes + m_xT.bytes;
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
    const auto seglen = static_cast<uint32_t>(m_seglen);
    const auto nseg = static_cast<uint32_t>(m_nseg);
    const auto nseg_pad = static_cast<uint32_t>(m_nseg_pad);
    const auto nfreq = static_cast<uint32_t>(m_nfreq);
    const auto* lens = m_lens.as<uint16_t>();
    const auto* off = m_lens_off.as<uint64_t>();
    const auto* nper = m_nper.as<uint32_t>();
    if (m_use_tma) {
        switch (m_nbins) {
        case 8: bf::launch_tma<8>(m_tmap, lens, off, nper, nfreq, nseg, nseg_pad, seglen, d_fold, m_status, s); break;
        case 16: bf::launch_tma<16>(m_tmap, lens, off, nper, nfreq, nseg, nseg_pad, seglen, d_fold, m_status, s); break;
        case 32: bf::launch_tma<32>(m_tmap, lens, off, nper, nfreq, nseg, nseg_pad, seglen, d_fold, m_status, s); break;
        case 64: bf::launch_tma<64>(m_tmap, lens, off, nper, nfreq, nseg, nseg_pad, seglen, d_fold, m_status, s); break;
        case 128: bf::launch_tma<128>(m_tmap, lens, off, nper, nfreq, nseg, nseg_pad, seglen, d_fold, m_status, s); break;
        default: fail(LK_ERR_INTERNAL, "unexpected nbins for the TMA brute fold");
        }
    } else {
        const size_t smem = 2ull * m_nbins * kWarp * sizeof(float);
        dim3 grid(nseg_pad / kWarp, nfreq);
        brute_fold_generic_kernel<<<grid, 2 * kWarp, smem, s>>>(
            m_xT.as<float>(), lens, off, nper, nfreq, nseg, nseg_pad, seglen,
            static_cast<uint32_t>(m_nbins), d_fold);
        LK_CUDA(cudaGetLastError());
    }
}

}  // namespace lk
