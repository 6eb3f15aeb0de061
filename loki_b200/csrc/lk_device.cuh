// Device helpers shared by the loki_b200 kernels.
//
// The phase and grid arithmetic below decides which fold row and which
// circular shift every output bin uses, so it must give the same bits as the
// reference's host code (compiled without FMA contraction). Each operation is
// spelled with an explicit round-to-nearest intrinsic, which nvcc never fuses,
// in the reference's evaluation order.
#pragma once

#include <cfloat>
#include <cstdint>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace lk::dev {

constexpr double kInvCval = 3.3356409519815204e-09;  // utils::kInvCval
constexpr double kFloatEps = 1e-6;                   // utils::kFloatEps

// Device status word bits (written with atomicOr, read by the host).
constexpr uint32_t kStatusWaitTimeout = 1u << 0;   // a bounded mbarrier wait gave up
constexpr uint32_t kStatusRunTooLong = 1u << 1;    // brute-fold run longer than 65535
constexpr uint32_t kStatusBadTable = 1u << 2;      // a table entry out of range
// Which brute-fold wait gave up (set together with kStatusWaitTimeout).
constexpr uint32_t kStatusFirstFull = 1u << 3;     // consumer, first stage
constexpr uint32_t kStatusFull = 1u << 4;          // consumer, later stages
constexpr uint32_t kStatusEmpty = 1u << 5;         // producer, stage reuse
constexpr uint32_t kStatusDrain = 1u << 6;         // producer, final loads

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double u2d(uint64_t x) { return __ull2double_rn(x); }

// psr_utils::get_phase_idx (lib/loki/psr_utils.hpp:32-49).
__device__ __forceinline__ float phase_idx(double proper_time, double freq, uint32_t nbins,
                                           double delay) {
    const double total_phase = dmul(dsub(proper_time, delay), freq);
    const double norm_phase = dsub(total_phase, floor(total_phase));
    const double nb = u2d(nbins);
    double iphase = dmul(norm_phase, nb);
    if (iphase >= nb) {
        iphase = 0.0;
    }
    return __double2float_rn(iphase);
}

// psr_utils::get_phase_idx_uint (lib/loki/psr_utils.hpp:53-63).
__device__ __forceinline__ uint32_t phase_idx_uint(double proper_time, double freq,
                                                   uint32_t nbins, double delay) {
    const float iphase = phase_idx(proper_time, freq, nbins, delay);
    uint32_t i = __float2uint_rz(__fadd_rn(iphase, 0.5f));
    if (i == nbins) {
        i = 0;
    }
    return i;
}

// psr_utils::get_param_val_at_idx (lib/loki/psr_utils.hpp:283-293).
__device__ __forceinline__ double param_val_at_idx(double vmin, double vmax, uint64_t count,
                                                   uint64_t i) {
    if (count <= 1) {
        return ddiv(dadd(vmax, vmin), 2.0);
    }
    const double dv_actual = ddiv(dsub(vmax, vmin), u2d(count));
    return dadd(vmin, dmul(dv_actual, dadd(u2d(i), 0.5)));
}

// psr_utils::get_nearest_idx_analytical (lib/loki/psr_utils.hpp:304-320).
__device__ __forceinline__ uint32_t nearest_idx(double val, double vmin, double vmax,
                                                uint64_t count) {
    if (count <= 1) {
        return 0;
    }
    const double raw_idx = ddiv(dmul(u2d(count), dsub(val, vmin)), dsub(vmax, vmin));
    const int idx = __double2int_rz(dadd(raw_idx, kFloatEps));
    if (idx < 0) {
        return 0;
    }
    if (idx >= static_cast<int>(count)) {
        return static_cast<uint32_t>(count - 1);
    }
    return static_cast<uint32_t>(idx);
}

// Integer circular shift used by every merge: round-half-up of the float
// phase, nbins wraps to 0 (lib/kernels.cpp:42-49,125-128).
__device__ __forceinline__ uint32_t shift_bins(float phase, uint32_t nbins) {
    uint32_t s = __float2uint_rz(__fadd_rn(phase, 0.5f));
    return s == nbins ? 0u : s;
}

// ---- storage conversions ------------------------------------------------
// Fold storage types: FP32, or BF16 (round to nearest even on store); every
// arithmetic operation is FP32.
template <class T> struct Store;
template <> struct Store<float> {
    __device__ __forceinline__ static float load(const float* p) { return __ldg(p); }
    __device__ __forceinline__ static void store(float* p, float v) { *p = v; }
    __device__ __forceinline__ static float from_float(float v) { return v; }
};
template <> struct Store<__nv_bfloat16> {
    __device__ __forceinline__ static float load(const __nv_bfloat16* p) {
        return __bfloat162float(__ldg(p));
    }
    __device__ __forceinline__ static void store(__nv_bfloat16* p, float v) {
        *p = __float2bfloat16_rn(v);
    }
    __device__ __forceinline__ static __nv_bfloat16 from_float(float v) {
        return __float2bfloat16_rn(v);
    }
};

}  // namespace lk::dev
