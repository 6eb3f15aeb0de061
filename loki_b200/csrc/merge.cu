// One hierarchical merge level of the FFA:
//
//   out[s, c, r, j] = in[2s,   tail(c), r, (j - st(c)) mod nbins]
//                   + in[2s+1, head(c), r, (j - sh(c)) mod nbins]
//
// for r in {E, V}. Freq-only plans (FFACoordFreq) use tail = head = idx and an
// unshifted tail (lib/kernels.cpp:118-146, 722-827); Taylor plans (FFACoord)
// shift both halves (lib/kernels.cpp:71-112, 829-940). Each output element is
// one FP32 add of the same two operands as the reference, so results are
// bit-identical.
//
// Work split: a warp per (segment, coordinate) row pair; lanes stride over
// the 2*nbins output elements, so every load and store instruction of a warp
// touches one contiguous (rotated) 128-byte span of a row.
#include "lk_device.cuh"
#include "lk_kernels.hpp"

namespace lk {

namespace {

constexpr int kWarp = 32;

struct CoordFreq {
    uint32_t idx;
    float shift;
};
struct CoordTaylor {
    uint32_t i_tail;
    float shift_tail;
    uint32_t i_head;
    float shift_head;
};

template <bool TAYLOR>
__device__ __forceinline__ void load_coord(const void* coords, uint64_t c, uint32_t nbins,
                                           uint32_t* it, uint32_t* st, uint32_t* ih,
                                           uint32_t* sh) {
    if constexpr (TAYLOR) {
        const CoordTaylor k = reinterpret_cast<const CoordTaylor*>(coords)[c];
        *it = k.i_tail;
        *ih = k.i_head;
        *st = dev::shift_bins(k.shift_tail, nbins);
        *sh = dev::shift_bins(k.shift_head, nbins);
    } else {
        const CoordFreq k = reinterpret_cast<const CoordFreq*>(coords)[c];
        *it = k.idx;
        *ih = k.idx;
        *st = 0;
        *sh = dev::shift_bins(k.shift, nbins);
    }
}

template <bool TAYLOR>
__global__ void merge_kernel(const float* __restrict__ in, float* __restrict__ out,
                             const void* __restrict__ coords, uint64_t ncur, uint64_t nprev,
                             uint64_t nseg, uint32_t nbins) {
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * (blockDim.x / kWarp);
    const uint64_t w0 = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp;
    const uint32_t lane = threadIdx.x % kWarp;
    const uint64_t total = nseg * ncur;
    const uint32_t row = 2 * nbins;
    for (uint64_t w = w0; w < total; w += nwarps) {
        const uint64_t s = w / ncur;
        const uint64_t c = w - s * ncur;
        uint32_t it, st, ih, sh;
        load_coord<TAYLOR>(coords, c, nbins, &it, &st, &ih, &sh);
        const float* tail = in + ((2 * s) * nprev + it) * row;
        const float* head = in + ((2 * s + 1) * nprev + ih) * row;
        float* o = out + w * row;
        for (uint32_t e = lane; e < row; e += kWarp) {
            const uint32_t r = e >= nbins ? nbins : 0;
            const uint32_t j = e - r;
            const uint32_t jt = j >= st ? j - st : j + nbins - st;
            const uint32_t jh = j >= sh ? j - sh : j + nbins - sh;
            o[e] = __fadd_rn(__ldg(tail + r + jt), __ldg(head + r + jh));
        }
    }
}

}  // namespace

void merge_level(const float* d_in, float* d_out, const void* d_coords, bool taylor,
                 uint64_t ncoords_cur, uint64_t ncoords_prev, uint64_t nsegments,
                 uint32_t nbins, cudaStream_t s) {
    const uint64_t total = ncoords_cur * nsegments;
    const unsigned threads = 256;
    const uint64_t want = (total + (threads / kWarp) - 1) / (threads / kWarp);
    const unsigned blocks = static_cast<unsigned>(want < 148ull * 64 ? want : 148ull * 64);
    if (taylor) {
        merge_kernel<true><<<blocks, threads, 0, s>>>(d_in, d_out, d_coords, ncoords_cur,
                                                      ncoords_prev, nsegments, nbins);
    } else {
        merge_kernel<false><<<blocks, threads, 0, s>>>(d_in, d_out, d_coords, ncoords_cur,
                                                       ncoords_prev, nsegments, nbins);
    }
    LK_CUDA(cudaGetLastError());
}

}  // namespace lk
