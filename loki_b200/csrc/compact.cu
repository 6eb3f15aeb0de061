// Ordered threshold compaction: keep (i, x[i]) for x[i] >= thr, in increasing
// i -- the order FFAFreqSweep produces (lib/ffa_freq_sweep.cpp:182-195).
// Three passes, no atomics, deterministic: per-tile counts, one exclusive scan
// of the counts, per-tile ordered scatter.
#include <cuda.h>

#include <mutex>

#include "lk_block.cuh"
#include "lk_device.cuh"
#include "lk_kernels.hpp"

namespace lk {

namespace {

constexpr uint32_t kThreads = 1024;
constexpr uint32_t kPerThread = 4;
constexpr uint32_t kTile = kThreads * kPerThread;

using blk::block_exclusive_scan;

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

// ---- allocation-free variant -------------------------------------------------
//
// For callers that cannot call cudaMalloc (or any allocating routine) at the
// point where they compact: e.g. a host framework that owns all device memory
// through its own pool and forbids direct allocations, or a latency-critical
// loop where an allocation, which may synchronise the device, is not allowed.
// The tile counts and offsets live in this file-scope device array instead of
// caller-provided scratch. Limits and sharing rules:
//   * n <= kNoAllocMaxN (2^28 scores): 65,536 tiles of 4,096, 768 KiB + 16 B
//     of device memory, held by every GPU that loads the library until exit;
//   * every call uses the same array, so calls whose work overlaps on the GPU
//     (e.g. on two streams) race and give wrong results; serialise them;
//   * the array keeps the previous call's contents; nothing needs clearing,
//     because each call writes every count and offset it later reads.
constexpr uint64_t kNoAllocMaxN = 1ull << 28;
constexpr uint64_t kNoAllocMaxTiles = kNoAllocMaxN / kTile;
// Same size rule as compact_scratch_bytes(), usable in a static_assert.
constexpr uint64_t compact_scratch_bytes_c(uint64_t n) {
    return ((n + kTile - 1) / kTile) * (sizeof(uint32_t) + sizeof(uint64_t)) + 16;
}
constexpr size_t kNoAllocScratchBytes =
    kNoAllocMaxTiles * (sizeof(uint32_t) + sizeof(uint64_t)) + 16;

static __device__ __align__(256) unsigned char g_compact_noalloc_scratch[kNoAllocScratchBytes];

namespace {

// Identifier of the calling thread's current CUDA context (cuCtxGetId), 0 if
// the driver cannot report one. A context created after cudaDeviceReset (or
// any teardown of the primary context) has a new identifier.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static const std::pair<GetCurrent, GetId> fns = [] {
        void* cur = nullptr;
        void* id = nullptr;
        cudaDriverEntryPointQueryResult q1{}, q2{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &cur, 12000, cudaEnableDefault, &q1) !=
                cudaSuccess ||
            q1 != cudaDriverEntryPointSuccess) {
            cur = nullptr;
        }
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &id, 12000, cudaEnableDefault, &q2) !=
                cudaSuccess ||
            q2 != cudaDriverEntryPointSuccess) {
            id = nullptr;
        }
        return std::make_pair(reinterpret_cast<GetCurrent>(cur), reinterpret_cast<GetId>(id));
    }();
    CUcontext ctx = nullptr;
    unsigned long long ident = 0;
    if (fns.first == nullptr || fns.second == nullptr || fns.first(&ctx) != CUDA_SUCCESS ||
        ctx == nullptr || fns.second(ctx, &ident) != CUDA_SUCCESS) {
        return 0;
    }
    return ident;
}

// Device address of g_compact_noalloc_scratch for the current device. In host
// code the symbol's name is only a host-side stand-in, so the address is
// looked up with the device current and cached per device together with the
// identifier of the context it was looked up in; a call in a different
// context (the device's context was reset and re-created) looks it up again.
void* noalloc_scratch_for_current_device() {
    static std::mutex mu;
    static void* addr[64] = {};
    static unsigned long long ctx_of[64] = {};
    int dev = -1;
    LK_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < 64, "device ordinal out of range");
    const unsigned long long ctx = current_context_id();  // 0 before the context exists
    std::lock_guard<std::mutex> lock(mu);
    if (addr[dev] == nullptr || ctx == 0 || ctx != ctx_of[dev]) {
        void* p = nullptr;
        LK_CUDA(cudaGetSymbolAddress(&p, g_compact_noalloc_scratch));  // creates the context if needed
        addr[dev] = p;
        ctx_of[dev] = current_context_id();
    }
    return addr[dev];
}

}  // namespace

void compact_ge_noalloc(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx,
                        float* d_vals, uint64_t max_out, uint64_t* d_count, cudaStream_t s) {
    if (n > kNoAllocMaxN) {
        fail(LK_ERR_INVALID_ARG,
             "lk_compact_ge_noalloc: n exceeds the static scratch limit of 2^28 scores");
    }
    static_assert(compact_scratch_bytes_c(kNoAllocMaxN) <= kNoAllocScratchBytes,
                  "static scratch too small");
    compact_ge(d_scores, n, thr, d_idx, d_vals, max_out, d_count,
               noalloc_scratch_for_current_device(), s);
}

void scan_counts(const uint32_t* d_counts, uint64_t n, uint64_t* d_offsets, uint64_t* d_total,
                 cudaStream_t s) {
    if (n == 0) {
        LK_CUDA(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), s));
        return;
    }
    tile_scan_kernel<<<1, kThreads, 0, s>>>(d_counts, n, d_offsets, d_total);
    LK_CUDA(cudaGetLastError());
}

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
