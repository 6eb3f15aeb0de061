// Coordinate resolution on the device: for every level >= 1 and every
// parameter cell of that level, the index of the parent cell in the previous
// level (tail and head halves) and the phase shift to apply before adding.
// One thread per output coordinate; FP64 throughout, bit-identical to the
// reference host code (see lk_device.cuh).
//
// Reference: core::ffa_taylor_resolve_freq_batch (lib/taylor_ffa.cpp:249-271),
// ffa_taylor_resolve_accel_batch / _jerk_batch (lib/taylor_ffa.cpp:19-188),
// FFAPlanBase::Impl::resolve_coordinates[_freq] (lib/plans.cpp:64-132).
#include <cmath>

#include "lk_device.cuh"
#include "lk_internal.hpp"

namespace lk {

namespace {

struct LevelArgs {
    uint64_t n_cur[3];
    uint64_t n_prev[3];
    double lim_min[3];
    double lim_max[3];
    double tsegment;  // ldexp(tseg_brute, level - 1)
    uint32_t nbins;
    uint64_t ncoords;
};

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

__global__ void resolve_freq_kernel(LevelArgs a, CoordFreq* __restrict__ out) {
    const uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (i >= a.ncoords) {
        return;
    }
    const double f_cur = dev::param_val_at_idx(a.lim_min[0], a.lim_max[0], a.n_cur[0], i);
    CoordFreq c;
    c.idx = dev::nearest_idx(f_cur, a.lim_min[0], a.lim_max[0], a.n_prev[0]);
    // The freq-only merge shifts the head half by the phase accumulated over
    // one previous-level segment: delta_t = tsegment.
    c.shift = dev::phase_idx(a.tsegment, f_cur, a.nbins, 0.0);
    out[i] = c;
}

// Accel (nparams = 2): coords are [accel, freq] row-major.
__device__ __forceinline__ void accel_half(const LevelArgs& a, uint64_t ia, uint64_t jf,
                                           double delta_t, uint32_t* idx, float* shift) {
    using namespace dev;
    const double half_delta_t_sq = dmul(dmul(0.5, delta_t), delta_t);
    const double a_cur = param_val_at_idx(a.lim_min[0], a.lim_max[0], a.n_cur[0], ia);
    const double v_new = dmul(a_cur, delta_t);
    const double d_new = dmul(a_cur, half_delta_t_sq);
    const uint64_t idx_a = nearest_idx(a_cur, a.lim_min[0], a.lim_max[0], a.n_prev[0]);
    const double f_cur = param_val_at_idx(a.lim_min[1], a.lim_max[1], a.n_cur[1], jf);
    const double f_new = dmul(f_cur, dsub(1.0, dmul(v_new, dev::kInvCval)));
    const double delay_rel = dmul(d_new, dev::kInvCval);
    *shift = phase_idx(delta_t, f_cur, a.nbins, delay_rel);
    const uint64_t idx_f = nearest_idx(f_new, a.lim_min[1], a.lim_max[1], a.n_prev[1]);
    *idx = static_cast<uint32_t>(idx_a * a.n_prev[1] + idx_f);
}

__global__ void resolve_accel_kernel(LevelArgs a, CoordTaylor* __restrict__ out) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (c >= a.ncoords) {
        return;
    }
    const uint64_t ia = c / a.n_cur[1];
    const uint64_t jf = c - ia * a.n_cur[1];
    // delta_t = (latter - 0.5) * tsegment; tail is latter = 0, head latter = 1.
    const double dt_tail = dev::dmul(-0.5, a.tsegment);
    const double dt_head = dev::dmul(0.5, a.tsegment);
    CoordTaylor r;
    accel_half(a, ia, jf, dt_tail, &r.i_tail, &r.shift_tail);
    accel_half(a, ia, jf, dt_head, &r.i_head, &r.shift_head);
    out[c] = r;
}

// Jerk (nparams = 3): coords are [jerk, accel, freq] row-major.
__device__ __forceinline__ void jerk_half(const LevelArgs& a, uint64_t ij, uint64_t ia,
                                          uint64_t jf, double delta_t, uint32_t* idx,
                                          float* shift) {
    using namespace dev;
    const double delta_t_sq = dmul(delta_t, delta_t);
    const double delta_t_cubed = dmul(delta_t_sq, delta_t);
    const double half_delta_t_sq = dmul(0.5, delta_t_sq);
    const double sixth_delta_t_cubed = ddiv(delta_t_cubed, 6.0);
    const double j_cur = param_val_at_idx(a.lim_min[0], a.lim_max[0], a.n_cur[0], ij);
    const double j_delta_t = dmul(j_cur, delta_t);
    const double half_j_delta_t_sq = dmul(dmul(0.5, j_cur), delta_t_sq);
    const double j_sixth_delta_t_cubed = dmul(j_cur, sixth_delta_t_cubed);
    const uint64_t idx_j = nearest_idx(j_cur, a.lim_min[0], a.lim_max[0], a.n_prev[0]);
    const double a_cur = param_val_at_idx(a.lim_min[1], a.lim_max[1], a.n_cur[1], ia);
    const double a_new = dadd(a_cur, j_delta_t);
    const double v_new = dadd(dmul(a_cur, delta_t), half_j_delta_t_sq);
    const double d_new = dadd(dmul(a_cur, half_delta_t_sq), j_sixth_delta_t_cubed);
    const uint64_t idx_a = nearest_idx(a_new, a.lim_min[1], a.lim_max[1], a.n_prev[1]);
    const double f_cur = param_val_at_idx(a.lim_min[2], a.lim_max[2], a.n_cur[2], jf);
    const double f_new = dmul(f_cur, dsub(1.0, dmul(v_new, dev::kInvCval)));
    const double delay_rel = dmul(d_new, dev::kInvCval);
    *shift = phase_idx(delta_t, f_cur, a.nbins, delay_rel);
    const uint64_t idx_f = nearest_idx(f_new, a.lim_min[2], a.lim_max[2], a.n_prev[2]);
    *idx = static_cast<uint32_t>(idx_j * a.n_prev[1] * a.n_prev[2] + idx_a * a.n_prev[2] +
                                 idx_f);
}

__global__ void resolve_jerk_kernel(LevelArgs a, CoordTaylor* __restrict__ out) {
    const uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (c >= a.ncoords) {
        return;
    }
    const uint64_t naf = a.n_cur[1] * a.n_cur[2];
    const uint64_t ij = c / naf;
    const uint64_t rem = c - ij * naf;
    const uint64_t ia = rem / a.n_cur[2];
    const uint64_t jf = rem - ia * a.n_cur[2];
    const double dt_tail = dev::dmul(-0.5, a.tsegment);
    const double dt_head = dev::dmul(0.5, a.tsegment);
    CoordTaylor r;
    jerk_half(a, ij, ia, jf, dt_tail, &r.i_tail, &r.shift_tail);
    jerk_half(a, ij, ia, jf, dt_head, &r.i_head, &r.shift_head);
    out[c] = r;
}

}  // namespace

void resolve_coords_device(const Plan& plan, void* d_coords, cudaStream_t stream) {
    require(!plan.offsets_overflow, "coordinate offsets exceed 32 bits");
    const uint32_t np = plan.nparams;
    if (np > 3) {
        fail(LK_ERR_UNSUPPORTED, "coordinate resolution supports nparams <= 3");
    }
    const size_t elem = (np == 1) ? sizeof(CoordFreq) : sizeof(CoordTaylor);
    // Level 0 is never resolved by the reference (lib/plans.cpp:77); zero it.
    LK_CUDA(cudaMemsetAsync(d_coords, 0, elem * plan.ncoords[0], stream));
    for (uint32_t l = 1; l < plan.n_levels; ++l) {
        LevelArgs a{};
        for (uint32_t i = 0; i < np; ++i) {
            a.n_cur[i] = plan.param_counts[l][i];
            a.n_prev[i] = plan.param_counts[l - 1][i];
            a.lim_min[i] = plan.lim_min(i);
            a.lim_max[i] = plan.lim_max(i);
        }
        a.tsegment = std::ldexp(plan.tseg_brute, static_cast<int>(l - 1));
        a.nbins = static_cast<uint32_t>(plan.cfg.nbins);
        a.ncoords = plan.ncoords[l];
        const unsigned threads = 256;
        const auto blocks = static_cast<unsigned>((a.ncoords + threads - 1) / threads);
        char* base = static_cast<char*>(d_coords) + elem * plan.ncoords_offsets[l];
        if (np == 1) {
            resolve_freq_kernel<<<blocks, threads, 0, stream>>>(a, reinterpret_cast<CoordFreq*>(base));
        } else if (np == 2) {
            resolve_accel_kernel<<<blocks, threads, 0, stream>>>(a, reinterpret_cast<CoordTaylor*>(base));
        } else {
            resolve_jerk_kernel<<<blocks, threads, 0, stream>>>(a, reinterpret_cast<CoordTaylor*>(base));
        }
        LK_CUDA(cudaGetLastError());
    }
}

}  // namespace lk
