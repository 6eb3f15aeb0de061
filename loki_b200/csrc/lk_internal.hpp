// Internal declarations shared by the loki_b200 host and device sources.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "loki_b200.h"

namespace lk {

// Exceptions never cross the C ABI: capi wrappers translate them to status
// codes and store the message for lk_last_error().
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

[[noreturn]] inline void fail(int status, const std::string& msg) { throw Error(status, msg); }
inline void require(bool ok, const std::string& msg) {
    if (!ok) {
        fail(LK_ERR_INVALID_ARG, msg);
    }
}

inline void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int st = (e == cudaErrorMemoryAllocation) ? LK_ERR_OOM : LK_ERR_CUDA;
        fail(st, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define LK_CUDA(call) ::lk::cuda_check((call), #call)

// utils::kCval / kInvCval / kFloatEps (lib/loki/utils.hpp:11-15 of the reference).
constexpr double kCval = 299792458.0;
constexpr double kInvCval = 3.3356409519815204e-09;
constexpr double kFloatEps = 1e-6;

// Host-side plan: configuration plus the per-level geometry of the reference
// FFAPlan (lib/plans.cpp:264-320).
struct Plan {
    lk_config cfg{};
    uint32_t nparams = 0;
    uint32_t n_levels = 0;
    uint64_t bseg_brute = 0;
    uint64_t bseg_ffa = 0;
    double tseg_brute = 0;
    double tseg_ffa = 0;
    std::vector<uint64_t> segment_lens, nsegments, ncoords;
    std::vector<double> tsegments;
    std::vector<uint32_t> ncoords_offsets;
    bool offsets_overflow = false;  // offsets or final ncoords past 32 bits (sizes-only plan)
    std::vector<std::vector<uint64_t>> param_counts;
    std::vector<std::vector<double>> dparams, dparams_actual;
    std::vector<uint32_t> widths;
    uint64_t buffer_size = 0;
    uint64_t coord_size = 0;

    double lim_min(uint32_t i) const { return cfg.param_limits[2 * i]; }
    double lim_max(uint32_t i) const { return cfg.param_limits[2 * i + 1]; }
    uint64_t fold_size(uint32_t level) const {
        return nsegments[level] * ncoords[level] * 2 * cfg.nbins;
    }
    uint64_t nfreq0() const { return param_counts[0][nparams - 1]; }
    // t_ref of the brute fold (lib/ffa.cpp:175-176).
    double t_ref0() const { return nparams == 1 ? 0.0 : tsegments[0] / 2.0; }
    std::vector<double> param_grid(uint32_t level, uint32_t iparam) const;
    std::vector<double> dparams_at(double tseg_cur, int kind) const;
    std::vector<double> branching_pattern(uint64_t ref_seg, bool conservative) const;
    std::vector<double> branching_pattern_cheby(uint64_t ref_seg) const;
    uint64_t prune_branch_max(bool conservative, int basis = 0) const;
};

Plan make_plan(const lk_config& cfg, bool sizes_only = false);
std::vector<uint32_t> box_width_trials(uint64_t nbins, double ducy_max, double wtsp);

// psr_utils::range_param (lib/loki/psr_utils.hpp:254-270).
std::vector<double> range_param(double vmin, double vmax, double dv);

// Device work, implemented in the .cu files. All enqueue on `stream`.
struct CoordTables;  // device coordinate tables of one plan
void resolve_coords_device(const Plan& plan, void* d_coords, cudaStream_t stream);

}  // namespace lk
