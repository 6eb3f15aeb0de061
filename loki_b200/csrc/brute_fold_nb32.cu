// Brute-fold kernel instantiation for nbins = 32.
#include "brute_fold_tma.cuh"

namespace lk::bf {
template void launch_tma<32>(const CUtensorMap&, const uint16_t*, const uint64_t*,
                              const uint32_t*, uint32_t, uint32_t, uint32_t, uint32_t, float*,
                              uint32_t*, cudaStream_t);
}  // namespace lk::bf
