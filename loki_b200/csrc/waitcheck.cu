// Check of the bounded device-side wait (lk_ptx.cuh::mbar_wait_bounded), the
// wait every pipelined kernel here uses on its mbarriers: one warp waits on a
// barrier that is either completed (one arrival) or never completed. In the
// second case the wait must give up after its time limit, set the timeout bit
// in the status word and return, leaving the context usable. No TMA or other
// asynchronous copy is issued, so nothing is in flight when the wait gives up.
#include "lk_device.cuh"
#include "lk_kernels.hpp"
#include "lk_ptx.cuh"

namespace lk {

namespace {

constexpr uint32_t kStatusSelfTest = 1u << 7;  // set with kStatusWaitTimeout by this check

__global__ void wait_check_kernel(uint64_t limit_ns, int complete, uint32_t* status) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        ptx::mbar_init(&bar, 1);
        ptx::fence_barrier_init();
    }
    __syncwarp();
    if (complete != 0 && threadIdx.x == 0) {
        ptx::mbar_arrive(&bar);
    }
    __syncwarp();
    ptx::mbar_wait_bounded(&bar, 0, status, dev::kStatusWaitTimeout | kStatusSelfTest, limit_ns);
}

}  // namespace

uint32_t wait_check(uint64_t limit_ns, bool complete, uint32_t* d_status, cudaStream_t s) {
    require(limit_ns >= 1000000ull && limit_ns <= ptx::kWaitLimitNs,
            "wait limit must lie in [1 ms, 0.5 s]");
    LK_CUDA(cudaMemsetAsync(d_status, 0, sizeof(uint32_t), s));
    wait_check_kernel<<<1, 32, 0, s>>>(limit_ns, complete ? 1 : 0, d_status);
    LK_CUDA(cudaGetLastError());
    uint32_t st = 0;
    LK_CUDA(cudaMemcpyAsync(&st, d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    return st;
}

}  // namespace lk
