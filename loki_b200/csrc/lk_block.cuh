// Block-wide primitives shared by the compaction (compact.cu) and pruning
// (prune.cu) kernels.
#pragma once

#include <cstdint>

namespace lk::blk {

// Exclusive scan of one uint32 per thread over the block (blockDim.x a
// multiple of 32, at most 1024). warp_sums: 32 words of shared memory. When
// total is non-null every thread receives the block sum there. Contains
// __syncthreads(): every thread of the block must call it.
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

}  // namespace lk::blk
