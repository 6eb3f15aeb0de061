// Ordered threshold compaction: keep (i, x[i]) for x[i] >= thr, in increasing
// i -- the order FFAFreqSweep produces (lib/ffa_freq_sweep.cpp:182-195).
// Three passes, no atomics, deterministic: per-tile counts, one exclusive scan
// of the counts, per-tile ordered scatter.
#include "lk_device.cuh"
#include "lk_kernels.hpp"

namespace lk {

namespace {

constexpr uint32_t kThreads = 1024;
constexpr uint32_t kPerThread = 4;
constexpr uint32_t kTile = kThreads * kPerThread;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums,
                                                         uint32_t* total) {
    const uint32_t lane = threadIdx.x % 32, warp = threadIdx.x / 32;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (static_cast<int>(lane) >= o) {
            x += t;
        }
    }
    if (lane == 31) {
        warp_sums[warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t nw = blockDim.x / 32;
        uint32_t y = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, y, o);
            if (static_cast<int>(lane) >= o) {
                y += t;
            }
        }
        if (lane < nw) {
            warp_sums[lane] = y;  // inclusive
        }
    }
    __syncthreads();
    const uint32_t before = (warp == 0 ? 0 : warp_sums[warp - 1]) + x - v;
    if (total != nullptr) {
        *total = warp_sums[blockDim.x / 32 - 1];
    }
    return before;
}

__global__ void tile_count_kernel(const float* __restrict__ x, uint64_t n, float thr,
                                  uint32_t* __restrict__ counts) {
    __shared__ uint32_t ws[32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTile + threadIdx.x * kPerThread;
    uint32_t c = 0;
#pragma unroll
    for (uint32_t q = 0; q < kPerThread; ++q) {
        const uint64_t i = base + q;
        c += (i < n && x[i] >= thr) ? 1u : 0u;
    }
    uint32_t total;
    block_exclusive_scan(c, ws, &total);
    if (threadIdx.x == 0) {
        counts[blockIdx.x] = total;
    }
}

// Single block: exclusive scan of the tile counts (chunks of kThreads).
__global__ void tile_scan_kernel(const uint32_t* __restrict__ counts, uint64_t ntiles,
                                 uint64_t* __restrict__ offsets, uint64_t* __restrict__ d_count) {
    __shared__ uint32_t ws[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) {
        carry = 0;
    }
    __syncthreads();
    for (uint64_t c0 = 0; c0 < ntiles; c0 += blockDim.x) {
        const uint64_t i = c0 + threadIdx.x;
        const uint32_t v = i < ntiles ? counts[i] : 0;
        uint32_t total;
        const uint32_t before = block_exclusive_scan(v, ws, &total);
        if (i < ntiles) {
            offsets[i] = carry + before;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry += total;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *d_count = carry;
    }
}

__global__ void tile_scatter_kernel(const float* __restrict__ x, uint64_t n, float thr,
                                    const uint64_t* __restrict__ offsets, uint32_t* __restrict__ idx,
                                    float* __restrict__ vals, uint64_t max_out) {
    __shared__ uint32_t ws[32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kTile + threadIdx.x * kPerThread;
    float v[kPerThread];
    uint32_t c = 0;
#pragma unroll
    for (uint32_t q = 0; q < kPerThread; ++q) {
        const uint64_t i = base + q;
        v[q] = i < n ? x[i] : 0.0f;
        c += (i < n && v[q] >= thr) ? 1u : 0u;
    }
    uint64_t pos = offsets[blockIdx.x] + block_exclusive_scan(c, ws, nullptr);
#pragma unroll
    for (uint32_t q = 0; q < kPerThread; ++q) {
        const uint64_t i = base + q;
        if (i < n && v[q] >= thr) {
            if (pos < max_out) {
                idx[pos] = static_cast<uint32_t>(i);
                vals[pos] = v[q];
            }
            ++pos;
        }
    }
}

}  // namespace

uint64_t compact_scratch_bytes(uint64_t n) {
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    return ntiles * (sizeof(uint32_t) + sizeof(uint64_t)) + 16;
}

void compact_ge(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx, float* d_vals,
                uint64_t max_out, uint64_t* d_count, void* d_scratch, cudaStream_t s) {
    require(n <= 0xffffffffULL, "compaction indices are 32-bit: n must be < 2^32");
    if (n == 0) {
        LK_CUDA(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), s));
        return;
    }
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    require(ntiles <= 0x7fffffffULL, "too many compaction tiles");
    auto* offsets = static_cast<uint64_t*>(d_scratch);
    auto* counts = reinterpret_cast<uint32_t*>(offsets + ntiles);
    tile_count_kernel<<<static_cast<unsigned>(ntiles), kThreads, 0, s>>>(d_scores, n, thr, counts);
    LK_CUDA(cudaGetLastError());
    tile_scan_kernel<<<1, kThreads, 0, s>>>(counts, ntiles, offsets, d_count);
    LK_CUDA(cudaGetLastError());
    tile_scatter_kernel<<<static_cast<unsigned>(ntiles), kThreads, 0, s>>>(
        d_scores, n, thr, offsets, d_idx, d_vals, max_out);
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
