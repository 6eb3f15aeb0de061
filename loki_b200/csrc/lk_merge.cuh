// Coordinate decoding shared by the merge kernels.
#pragma once

#include <cstdint>

#include "lk_device.cuh"

namespace lk {

// FFACoordFreq / FFACoord (include/loki/common/coord.hpp:15-25 of the reference).
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
static_assert(sizeof(CoordFreq) == 8 && sizeof(CoordTaylor) == 16, "coord layout");

// Parent rows and integer circular shifts of one output coordinate.
struct MergeCoord {
    uint32_t it, ih, st, sh;
};

template <bool TAYLOR>
__device__ __forceinline__ MergeCoord load_merge_coord(const void* coords, uint64_t c,
                                                       uint32_t nbins) {
    MergeCoord m;
    if constexpr (TAYLOR) {
        const CoordTaylor k = reinterpret_cast<const CoordTaylor*>(coords)[c];
        m.it = k.i_tail;
        m.ih = k.i_head;
        m.st = dev::shift_bins(k.shift_tail, nbins);
        m.sh = dev::shift_bins(k.shift_head, nbins);
    } else {
        const CoordFreq k = reinterpret_cast<const CoordFreq*>(coords)[c];
        m.it = k.idx;
        m.ih = k.idx;
        m.st = 0;
        m.sh = dev::shift_bins(k.shift, nbins);
    }
    return m;
}

}  // namespace lk
