// Pruning leaf step on the GPU: seed, branch, resolve, shift-add, score and
// filter, transform, and the world-tree update of one pruning level, for
// Taylor-basis searches with nparams 2 (accel) or 3 (jerk).
//
// Reference: PruneImpl::initialize / execute_iteration_batched
// (lib/prune.cpp:181-226,429-620) over the Taylor PruneDPFuncts
// (lib/dynamic.cpp:155-310, lib/taylor.cpp:24-314,492-619,881-1005,
// 1197-1257), kernels::shift_add_linear_batch (lib/kernels.cpp:1328-1355),
// score_and_filter_max_with_cache (lib/score.cpp:213-259) and the WorldTree
// circular buffer (lib/world_tree.cpp:237-276,361-422,557-669).
//
// The reference walks a level in batches of `batch_size` parents and, per
// batch, branches, scores, filters with the current threshold and adds the
// survivors to the world tree, whose overload pruning can raise that
// threshold for the batches that follow. Here, the work that does not depend
// on the threshold is done for the whole level at once:
//   1. branch_count / scan / branch_emit: every parent's children, in parent
//      order (the reference's concatenated batch outputs);
//   2. leaf_kernel: resolve, shift-add and max-width S/N of every child, one
//      child per thread for the FP64 and scoring parts and one warp per
//      child for the fold rows; folds are kept only for children at or above
//      the level's starting threshold, the lowest threshold any batch uses.
// The threshold-dependent part keeps the reference's batch semantics exactly:
// the host replays the WorldTree bookkeeping (sizes, space left, batch
// boundaries at the circular buffer's wrap) from per-batch pass counts, and
// the device holds the write region as an ordered list of (child, score).
// Runs of batches that fit are appended with one ordered compaction; a batch
// that overflows runs the reference's overload step on the device (exact
// order statistics by radix select, threshold = max(current, next above the
// k-th, next above the selected median), prune the list by score >
// threshold, append the batch's children >= threshold up to the space left).
// At the end of the level the surviving children are transformed and
// gathered into the other of two tree buffers at the reference's physical
// slots, so the next level's batch boundaries match the reference's.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "lk_block.cuh"
#include "lk_device.cuh"
#include "lk_prune.hpp"
#include "lk_ptx.cuh"
#include "lk_score.cuh"

namespace lk {

namespace {

constexpr uint32_t kWarp = 32;
constexpr uint32_t kScanThreads = 1024;
constexpr uint32_t kScanPer = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanPer;

// Status bits (beside those of lk_device.cuh).
constexpr uint32_t kStatusBranchMax = 1u << 8;   // a parameter needs > branch_max points
constexpr uint32_t kStatusZeroStep = 1u << 9;    // non-positive step size when branching
constexpr uint32_t kStatusBranchCount = 1u << 10;  // children of one parent exceed 2^32-1

// Grid geometry of one search, by value in kernel arguments.
struct LeafGeom {
    uint32_t np;       // 2 (accel, freq) or 3 (jerk, accel, freq)
    uint32_t nbins;
    uint32_t ls;       // doubles per leaf: (np + 2) * 2
    uint32_t n_accel;  // final FFA level counts used by resolve
    uint32_t n_freq;
    double eta;
    double a_min, a_max, f_min, f_max;
    uint64_t branch_max;
    uint32_t basis;    // 0 Taylor, 1 Chebyshev
};

// Per-parameter branching of one parent: values base + i * step (i < count)
// when `split`, else the parent value itself.
struct ParamBranch {
    double cur, first, act, dparam;
    uint32_t count;
    bool split;
};

// poly_taylor_branch_{accel,jerk}_batch steps and shifts (lib/taylor.cpp:
// 64-85, 199-227), then branch_one_param_padded / branch_param_padded
// (lib/loki/psr_utils.hpp:189-211, lib/psr_utils.cpp:226-259). Plain
// double operators are IEEE round-to-nearest here (the library is built
// with -fmad=false), in the reference's association.
__device__ void branch_params(const double* lf, double dt, const LeafGeom& g, ParamBranch* pb,
                              uint32_t* status) {
    const double nbins_d = static_cast<double>(g.nbins);
    const double dphi = g.eta / nbins_d;
    const double dt2 = dt * dt;
    const double inv_dt = 1.0 / dt;
    const double inv_dt2 = inv_dt * inv_dt;
    const double f0 = lf[(g.np + 1) * 2];
    const double dfactor = kCval / f0;
    double sig_new[3], shift[3];
    if (g.basis == 1) {
        // poly_chebyshev_branch_{accel,jerk}_batch (lib/chebyshev.cpp:
        // 530-551, 677-702): one step dphi C / f0 for every coefficient,
        // shift |sigma_cur - step| nbins / (C / f0).
        const double base_step = dphi * dfactor;
        const double inv_base = nbins_d / dfactor;
        for (uint32_t k = 0; k < g.np; ++k) {
            sig_new[k] = base_step;
            shift[k] = fabs(lf[2 * k + 1] - base_step) * inv_base;
        }
    } else if (g.np == 2) {
        sig_new[0] = dphi * dfactor * 4.0 * inv_dt2;
        sig_new[1] = dphi * dfactor * 1.0 * inv_dt;
        shift[0] = fabs(lf[1] - sig_new[0]) * dt2 * nbins_d / (4.0 * dfactor);
        shift[1] = fabs(lf[3] - sig_new[1]) * dt * nbins_d / (1.0 * dfactor);
    } else {
        const double dt3 = dt2 * dt;
        const double inv_dt3 = inv_dt2 * inv_dt;
        sig_new[0] = dphi * dfactor * 24.0 * inv_dt3;
        sig_new[1] = dphi * dfactor * 4.0 * inv_dt2;
        sig_new[2] = dphi * dfactor * 1.0 * inv_dt;
        shift[0] = fabs(lf[1] - sig_new[0]) * dt3 * nbins_d / (24.0 * dfactor);
        shift[1] = fabs(lf[3] - sig_new[1]) * dt2 * nbins_d / (4.0 * dfactor);
        shift[2] = fabs(lf[5] - sig_new[2]) * dt * nbins_d / (1.0 * dfactor);
    }
    for (uint32_t k = 0; k < g.np; ++k) {
        ParamBranch& b = pb[k];
        const double cur = lf[2 * k], sig_cur = lf[2 * k + 1];
        b.cur = cur;
        if (!(shift[k] >= (g.eta - kFloatEps))) {
            b.split = false;
            b.count = 1;
            b.dparam = sig_cur;
            b.first = cur;
            b.act = 0.0;
            continue;
        }
        b.split = true;
        if (sig_cur <= 1e-12 || sig_new[k] <= 1e-12) {  // utils::kZeroEps
            atomicOr(status, kStatusZeroStep);
            b.count = 1;
            b.dparam = sig_cur;
            b.first = cur;
            b.act = 0.0;
            continue;
        }
        const double ratio = sig_cur / sig_new[k];
        const double c = ceil(ratio - kFloatEps);
        uint64_t num = c < 1.0 ? 1 : static_cast<uint64_t>(c);
        if (num > g.branch_max) {
            atomicOr(status, kStatusBranchMax);
            num = 1;
        }
        const double act = sig_cur / static_cast<double>(num);
        const double parent_min = cur - (sig_cur / 2.0);
        b.first = parent_min + (act / 2.0);
        b.act = act;
        b.dparam = act;
        b.count = static_cast<uint32_t>(num);
    }
}

__device__ __forceinline__ double branch_value(const ParamBranch& b, uint32_t i) {
    return b.split ? b.first + (static_cast<double>(i) * b.act) : b.cur;
}

__global__ void branch_count_kernel(const double* __restrict__ tree_leaves, uint64_t head,
                                    uint64_t cap, uint64_t n, double dt, LeafGeom g,
                                    uint32_t* __restrict__ counts, uint32_t* status) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const double* lf = tree_leaves + ((head + i) % cap) * g.ls;
    ParamBranch pb[3];
    branch_params(lf, dt, g, pb, status);
    uint64_t prod = 1;
    for (uint32_t k = 0; k < g.np; ++k) {
        prod *= pb[k].count;
    }
    if (prod > 0xffffffffull) {
        atomicOr(status, kStatusBranchCount);
        prod = 1;
    }
    counts[i] = static_cast<uint32_t>(prod);
}

// Children of parent i at offsets[i]..: Cartesian product with the highest
// derivative outermost (lib/taylor.cpp:131-157, 282-311); d0 and f0 copied
// from the parent.
__global__ void branch_emit_kernel(const double* __restrict__ tree_leaves, uint64_t head,
                                   uint64_t cap, uint64_t n, double dt, LeafGeom g,
                                   const uint64_t* __restrict__ offsets,
                                   double* __restrict__ out, uint32_t* __restrict__ parent,
                                   uint32_t* status) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    const double* lf = tree_leaves + ((head + i) % cap) * g.ls;
    ParamBranch pb[3];
    branch_params(lf, dt, g, pb, status);
    uint64_t o = offsets[i];
    const uint32_t c2 = g.np == 3 ? pb[2].count : 1;
    for (uint32_t a = 0; a < pb[0].count; ++a) {
        const double va = branch_value(pb[0], a);
        for (uint32_t b = 0; b < pb[1].count; ++b) {
            const double vb = branch_value(pb[1], b);
            for (uint32_t c = 0; c < c2; ++c) {
                double* d = out + o * g.ls;
                d[0] = va;
                d[1] = pb[0].dparam;
                d[2] = vb;
                d[3] = pb[1].dparam;
                if (g.np == 3) {
                    d[4] = branch_value(pb[2], c);
                    d[5] = pb[2].dparam;
                }
                for (uint32_t q = 2 * g.np; q < g.ls; ++q) {
                    d[q] = lf[q];
                }
                parent[o] = static_cast<uint32_t>(i);
                ++o;
            }
        }
    }
}

// core::poly_taylor_seed (lib/taylor.cpp:1197-1257): leaf (ia, jf) of the
// final FFA level grid, accel-major.
__global__ void seed_kernel(LeafGeom g, double dp0, double dp1, double dfreq, double* out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t n = static_cast<uint64_t>(g.n_accel) * g.n_freq;
    if (i >= n) {
        return;
    }
    const uint64_t ia = i / g.n_freq, jf = i - ia * g.n_freq;
    const double accel = dev::param_val_at_idx(g.a_min, g.a_max, g.n_accel, ia);
    const double freq = dev::param_val_at_idx(g.f_min, g.f_max, g.n_freq, jf);
    double* o = out + i * g.ls;
    const uint32_t np = g.np;
    const double dps[2] = {dp0, dp1};
    for (uint32_t j = 0; j + 1 < np; ++j) {
        o[j * 2 + 0] = 0;
        o[j * 2 + 1] = dps[j];
    }
    o[(np - 2) * 2 + 0] = accel;
    o[(np - 1) * 2 + 0] = 0;
    o[(np - 1) * 2 + 1] = dfreq * (kCval / freq);
    o[np * 2 + 0] = 0;
    o[np * 2 + 1] = 0;
    o[(np + 1) * 2 + 0] = freq;
    o[(np + 1) * 2 + 1] = 0;
}

// poly_taylor_to_cheby_{accel,jerk}_batch (lib/chebyshev.cpp:58-93,145-189),
// in place, ts = coord_init.second.
__device__ __forceinline__ void taylor_to_cheby_leaf(double* lf, uint32_t np, double ts) {
    const double ts2 = ts * ts;
    if (np == 2) {
        const double w2_2 = (ts2 / 2.0) * 0.5;
        const double d2v = lf[0], d2e = lf[1], d1v = lf[2], d1e = lf[3], d0v = lf[4], d0e = lf[5];
        lf[0] = d2v * w2_2;
        lf[2] = d1v * ts;
        lf[4] = d0v + (d2v * w2_2);
        const double e2 = d2e * w2_2;
        const double e1_ts = d1e * ts;
        lf[1] = e2;
        lf[3] = e1_ts;
        lf[5] = __dsqrt_rn((d0e * d0e) + (e2 * e2));
    } else {
        const double ts3 = ts2 * ts;
        const double w3_3 = (ts3 / 6.0) * 0.25;
        const double w2_2 = (ts2 / 2.0) * 0.5;
        const double w3_1 = (ts3 / 6.0) * 0.75;
        const double d3v = lf[0], d3e = lf[1], d2v = lf[2], d2e = lf[3], d1v = lf[4], d1e = lf[5],
                     d0v = lf[6], d0e = lf[7];
        lf[0] = d3v * w3_3;
        lf[2] = d2v * w2_2;
        lf[4] = (d1v * ts) + (d3v * w3_1);
        lf[6] = d0v + (d2v * w2_2);
        const double e3_3 = d3e * w3_3;
        const double e2_2 = d2e * w2_2;
        const double e3_1 = d3e * w3_1;
        const double e1_ts = d1e * ts;
        lf[1] = e3_3;
        lf[3] = e2_2;
        lf[5] = __dsqrt_rn((e1_ts * e1_ts) + (e3_1 * e3_1));
        lf[7] = __dsqrt_rn((d0e * d0e) + (e2_2 * e2_2));
    }
}

// poly_cheby_to_taylor_{accel,jerk}_batch (lib/chebyshev.cpp:21-56,95-143),
// in place, ts = coord_report.second.
__device__ __forceinline__ void cheby_to_taylor_leaf(double* lf, uint32_t np, double ts) {
    const double inv_ts = 1.0 / ts;
    const double inv_ts2 = inv_ts * inv_ts;
    if (np == 2) {
        const double w2_2 = 4.0 * inv_ts2;
        const double w1_1 = inv_ts;
        const double a2v = lf[0], a2e = lf[1], a1v = lf[2], a1e = lf[3], a0v = lf[4], a0e = lf[5];
        lf[0] = a2v * w2_2;
        lf[2] = a1v * w1_1;
        lf[4] = a0v - a2v;
        lf[1] = a2e * w2_2;
        lf[3] = a1e * w1_1;
        lf[5] = __dsqrt_rn((a0e * a0e) + (a2e * a2e));
    } else {
        const double inv_ts3 = inv_ts2 * inv_ts;
        const double w3_3 = 24.0 * inv_ts3;
        const double w2_2 = 4.0 * inv_ts2;
        const double w1_1 = inv_ts;
        const double w3_1 = 3.0 * inv_ts;
        const double a3v = lf[0], a3e = lf[1], a2v = lf[2], a2e = lf[3], a1v = lf[4], a1e = lf[5],
                     a0v = lf[6], a0e = lf[7];
        lf[0] = a3v * w3_3;
        lf[2] = a2v * w2_2;
        lf[4] = (a1v * w1_1) - (a3v * w3_1);
        lf[6] = a0v - a2v;
        const double e3_3 = a3e * w3_3;
        const double e2_2 = a2e * w2_2;
        const double e1_1 = a1e * w1_1;
        const double e3_1 = a3e * w3_1;
        lf[1] = e3_3;
        lf[3] = e2_2;
        lf[5] = __dsqrt_rn((e1_1 * e1_1) + (e3_1 * e3_1));
        lf[7] = __dsqrt_rn((a0e * a0e) + (a2e * a2e));
    }
}

__global__ void basis_convert_kernel(double* __restrict__ leaves, uint64_t n, uint32_t np,
                                     double ts, int to_cheby) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    double* lf = leaves + i * (np + 2) * 2;
    if (to_cheby) {
        taylor_to_cheby_leaf(lf, np, ts);
    } else {
        cheby_to_taylor_leaf(lf, np, ts);
    }
}

// ---- exclusive scan of uint32 counts into uint64 offsets -------------------

__global__ void scan_tile_sums_kernel(const uint32_t* __restrict__ x, uint64_t n,
                                      uint32_t* __restrict__ sums) {
    __shared__ uint32_t ws[32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    uint32_t c = 0;
#pragma unroll
    for (uint32_t q = 0; q < kScanPer; ++q) {
        c += (base + q < n) ? x[base + q] : 0u;
    }
    uint32_t total;
    blk::block_exclusive_scan(c, ws, &total);
    if (threadIdx.x == 0) {
        sums[blockIdx.x] = total;
    }
}

// Single block: exclusive scan of per-tile sums (uint32 each) into uint64.
__global__ void scan_tiles_kernel(const uint32_t* __restrict__ sums, uint64_t ntiles,
                                  uint64_t* __restrict__ offs, uint64_t* __restrict__ d_total) {
    __shared__ uint32_t ws[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0) {
        carry = 0;
    }
    __syncthreads();
    for (uint64_t c0 = 0; c0 < ntiles; c0 += blockDim.x) {
        const uint64_t i = c0 + threadIdx.x;
        const uint32_t v = i < ntiles ? sums[i] : 0;
        uint32_t total;
        const uint32_t before = blk::block_exclusive_scan(v, ws, &total);
        if (i < ntiles) {
            offs[i] = carry + before;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry += total;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *d_total = carry;
    }
}

__global__ void scan_apply_kernel(const uint32_t* __restrict__ x, uint64_t n,
                                  const uint64_t* __restrict__ tile_offs,
                                  uint64_t* __restrict__ out) {
    __shared__ uint32_t ws[32];
    const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    uint32_t v[kScanPer];
    uint32_t c = 0;
#pragma unroll
    for (uint32_t q = 0; q < kScanPer; ++q) {
        v[q] = (base + q < n) ? x[base + q] : 0u;
        c += v[q];
    }
    uint64_t pos = tile_offs[blockIdx.x] + blk::block_exclusive_scan(c, ws, nullptr);
#pragma unroll
    for (uint32_t q = 0; q < kScanPer; ++q) {
        if (base + q < n) {
            out[base + q] = pos;
        }
        pos += v[q];
    }
}

// Child offsets at the batch boundaries (parent index -> first child).
__global__ void batch_child_starts_kernel(const uint64_t* __restrict__ offsets, uint64_t n,
                                          const uint64_t* __restrict__ d_total,
                                          const uint64_t* __restrict__ parent_starts,
                                          uint64_t nb1, uint64_t* __restrict__ child_starts) {
    const uint64_t b = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (b < nb1) {
        const uint64_t p = parent_starts[b];
        child_starts[b] = p < n ? offsets[p] : *d_total;
    }
}

// ---- resolve + shift-add + score ------------------------------------------

// poly_taylor_resolve_{accel,jerk}_batch (lib/taylor.cpp:492-619).
struct ResolveConsts {
    double dt;          // dt_add - dt_init
    double dt_add;      // t_add - t_cur (jerk's a_new)
    double half_dt2;
    double sixth_dt3;   // jerk only
    // Chebyshev (lib/chebyshev.cpp:961-1097)
    uint32_t basis;
    double dt2, dt3;    // dt_add^k - dt_init^k
    double inv_ts, inv_ts2, inv_ts3;
};

__device__ __forceinline__ void resolve_leaf(const double* lf, const LeafGeom& g,
                                             const ResolveConsts& rc, uint32_t* pidx,
                                             float* phase) {
    if (rc.basis == 1) {
        // poly_chebyshev_resolve_{accel,jerk}_batch
        double a_new, delta_v, delta_d, f0;
        if (g.np == 2) {
            const double alpha_2 = lf[0], alpha_1 = lf[2];
            f0 = lf[6];
            a_new = 4.0 * alpha_2 * rc.inv_ts2;
            delta_v = 4.0 * alpha_2 * rc.inv_ts2 * rc.dt;
            delta_d = (alpha_1 * rc.inv_ts * rc.dt) + (2.0 * alpha_2 * rc.inv_ts2 * rc.dt2);
        } else {
            const double alpha_3 = lf[0], alpha_2 = lf[2], alpha_1 = lf[4];
            f0 = lf[8];
            a_new = (4.0 * alpha_2 * rc.inv_ts2) + (24.0 * alpha_3 * rc.dt_add * rc.inv_ts3);
            delta_v = ((4.0 * alpha_2 * rc.inv_ts2) * rc.dt) +
                      ((12.0 * alpha_3 * rc.inv_ts3) * rc.dt2);
            delta_d = ((alpha_1 - (3.0 * alpha_3)) * rc.inv_ts * rc.dt) +
                      ((2.0 * alpha_2 * rc.inv_ts2) * rc.dt2) +
                      ((4.0 * alpha_3 * rc.inv_ts3) * rc.dt3);
        }
        const double f_new = f0 * (1.0 - (delta_v * kInvCval));
        const double delay_rel = delta_d * kInvCval;
        *phase = dev::phase_idx(rc.dt, f0, g.nbins, delay_rel);
        const uint32_t ia = dev::nearest_idx(a_new, g.a_min, g.a_max, g.n_accel);
        const uint32_t jf = dev::nearest_idx(f_new, g.f_min, g.f_max, g.n_freq);
        *pidx = ia * g.n_freq + jf;
        return;
    }
    if (g.np == 2) {
        const double a_cur = lf[0], v_cur = lf[2], f0 = lf[6];
        const double a_new = a_cur;
        const double delta_v = a_cur * rc.dt;
        const double delta_d = (v_cur * rc.dt) + (a_cur * rc.half_dt2);
        const double f_new = f0 * (1.0 - (delta_v * kInvCval));
        const double delay_rel = delta_d * kInvCval;
        const uint32_t ia = dev::nearest_idx(a_new, g.a_min, g.a_max, g.n_accel);
        const uint32_t jf = dev::nearest_idx(f_new, g.f_min, g.f_max, g.n_freq);
        *pidx = ia * g.n_freq + jf;
        *phase = dev::phase_idx(rc.dt, f0, g.nbins, delay_rel);
    } else {
        const double j_cur = lf[0], a_cur = lf[2], v_cur = lf[4], f0 = lf[8];
        const double a_new = a_cur + (j_cur * rc.dt_add);
        const double delta_v = (a_cur * rc.dt) + (j_cur * rc.half_dt2);
        const double delta_d = (v_cur * rc.dt) + (a_cur * rc.half_dt2) + (j_cur * rc.sixth_dt3);
        const double f_new = f0 * (1.0 - (delta_v * kInvCval));
        const double delay_rel = delta_d * kInvCval;
        *phase = dev::phase_idx(rc.dt, f0, g.nbins, delay_rel);
        const uint32_t ia = dev::nearest_idx(a_new, g.a_min, g.a_max, g.n_accel);
        const uint32_t jf = dev::nearest_idx(f_new, g.f_min, g.f_max, g.n_freq);
        *pidx = ia * g.n_freq + jf;
    }
}

// Orderable uint32 key of a float: larger float <-> larger key.
__device__ __forceinline__ uint32_t fkey(float x) {
    const uint32_t u = __float_as_uint(x);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// One block scores T consecutive children. Phase 0 (thread per child):
// resolve in FP64. Phase 1 (warp per child): tree fold + rotated FFA fold,
// normalised into shared memory (kernels::shift_add_linear_with_buffer,
// lib/kernels.cpp:118-146: out[j] = tree[j] + ffa[(j - s) mod nbins]).
// Phase 2 (thread per child): the reference's sequential prefix sum and
// width maxima. Phase 3 (warp per child): children scoring at or above
// thr_keep get their fold written for the world tree.
// One tile of blockDim.x children starting at c0 (< n); rows: the block's
// dynamic shared memory (blockDim.x rows of rs floats + 4 blockDim.x words).
// Ends with warps still writing kept folds: a caller that runs another tile
// synchronises the block first.
template <int NW, int NB>
__device__ __forceinline__ void leaf_tile(float* rows, uint64_t c0, const double* __restrict__ leaves,
                                          const uint32_t* __restrict__ parent, uint64_t n,
                                          const float* __restrict__ tree_folds, uint64_t head,
                                          uint64_t cap, const float* __restrict__ ffa_seg,
                                          const LeafGeom& g, const ResolveConsts& rc, uint32_t rs,
                                          const ScoreParams& sp, float thr_keep,
                                          float* __restrict__ scores, float* __restrict__ folds_out,
                                          uint32_t* __restrict__ minmax) {
    const uint32_t T = blockDim.x;
    uint32_t* s_pidx = reinterpret_cast<uint32_t*>(rows + static_cast<size_t>(T) * rs);
    uint32_t* s_shift = s_pidx + T;
    uint32_t* s_tree = s_shift + T;
    uint32_t* s_keep = s_tree + T;
    __shared__ uint32_t s_min, s_max;
    const uint32_t nhere = static_cast<uint32_t>((n - c0) < T ? (n - c0) : T);
    const uint32_t nb = g.nbins;
    if (threadIdx.x == 0) {
        s_min = 0xffffffffu;
        s_max = 0u;
    }
    if (threadIdx.x < nhere) {
        const uint64_t c = c0 + threadIdx.x;
        uint32_t pidx;
        float phase;
        resolve_leaf(leaves + c * g.ls, g, rc, &pidx, &phase);
        s_pidx[threadIdx.x] = pidx;
        s_shift[threadIdx.x] = dev::shift_bins(phase, nb);
        s_tree[threadIdx.x] = static_cast<uint32_t>((head + parent[c]) % cap);
    }
    __syncthreads();
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    if constexpr (NB > 0) {
        // nbins == NB, a multiple of 32: masked rotation, no bounds test; a
        // warp takes PB children at a time with all their row loads in flight
        constexpr int NJ = NB / static_cast<int>(kWarp);
        constexpr int PB = NB == 128 ? 2 : 4;
        for (uint32_t p0 = warp * PB; p0 < nhere; p0 += (T / kWarp) * PB) {
            float te[PB][NJ], tv[PB][NJ], he[PB][NJ], hv[PB][NJ];
#pragma unroll
            for (int q = 0; q < PB; ++q) {
                // children past nhere load the block's first child (in range, unused)
                const uint32_t p = p0 + q < nhere ? p0 + q : p0;
                const float* tail = tree_folds + static_cast<uint64_t>(s_tree[p]) * 2 * NB;
                const float* hd = ffa_seg + static_cast<uint64_t>(s_pidx[p]) * 2 * NB;
                const uint32_t s = s_shift[p];
#pragma unroll
                for (int u = 0; u < NJ; ++u) {
                    const uint32_t j = lane + kWarp * u;
                    const float* ph = hd + ((j - s) & (NB - 1));
                    te[q][u] = __ldg(tail + j);
                    tv[q][u] = __ldg(tail + NB + j);
                    he[q][u] = __ldg(ph);
                    hv[q][u] = __ldg(ph + NB);
                }
            }
#pragma unroll
            for (int q = 0; q < PB; ++q) {
                if (p0 + q < nhere) {
                    float* dst = rows + static_cast<size_t>(p0 + q) * rs;
#pragma unroll
                    for (int u = 0; u < NJ; ++u) {
                        dst[lane + kWarp * u] =
                            sc::normalise(__fadd_rn(te[q][u], he[q][u]), __fadd_rn(tv[q][u], hv[q][u]));
                    }
                }
            }
        }
    } else {
        for (uint32_t p = warp; p < nhere; p += T / kWarp) {
            const float* tail = tree_folds + static_cast<uint64_t>(s_tree[p]) * 2 * nb;
            const float* hd = ffa_seg + static_cast<uint64_t>(s_pidx[p]) * 2 * nb;
            const uint32_t s = s_shift[p];
            float* dst = rows + static_cast<size_t>(p) * rs;
            for (uint32_t j = lane; j < nb; j += kWarp) {
                const uint32_t jh = j >= s ? j - s : j + nb - s;
                const float e = __fadd_rn(__ldg(tail + j), __ldg(hd + jh));
                const float v = __fadd_rn(__ldg(tail + nb + j), __ldg(hd + nb + jh));
                dst[j] = sc::normalise(e, v);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const uint64_t c = c0 + threadIdx.x;
        float score;
        sc::score_row_any<NB, NW>(rows + static_cast<size_t>(threadIdx.x) * rs, nb, 1.0f, sp,
                                  LK_SCORE_MAX, &score);
        scores[c] = score;
        s_keep[threadIdx.x] = score >= thr_keep ? 1u : 0u;
        const uint32_t k = fkey(score);
        atomicMin(&s_min, k);
        atomicMax(&s_max, k);
    }
    __syncthreads();
    if (threadIdx.x == 0 && nhere > 0) {
        atomicMin(&minmax[0], s_min);
        atomicMax(&minmax[1], s_max);
    }
    for (uint32_t p = warp; p < nhere; p += T / kWarp) {
        if (s_keep[p] == 0) {
            continue;
        }
        const float* tail = tree_folds + static_cast<uint64_t>(s_tree[p]) * 2 * nb;
        const float* hd = ffa_seg + static_cast<uint64_t>(s_pidx[p]) * 2 * nb;
        const uint32_t s = s_shift[p];
        float* o = folds_out + (c0 + p) * 2 * nb;
        for (uint32_t j = lane; j < nb; j += kWarp) {
            const uint32_t jh = j >= s ? j - s : j + nb - s;
            o[j] = __fadd_rn(__ldg(tail + j), __ldg(hd + jh));
            o[nb + j] = __fadd_rn(__ldg(tail + nb + j), __ldg(hd + nb + jh));
        }
    }
}

template <int NW, int NB>
__global__ void leaf_kernel(const double* __restrict__ leaves, const uint32_t* __restrict__ parent,
                            uint64_t n, const float* __restrict__ tree_folds, uint64_t head,
                            uint64_t cap, const float* __restrict__ ffa_seg, LeafGeom g,
                            ResolveConsts rc, uint32_t rs, ScoreParams sp, float thr_keep,
                            float* __restrict__ scores, float* __restrict__ folds_out,
                            uint32_t* __restrict__ minmax) {
    extern __shared__ float rows[];
    leaf_tile<NW, NB>(rows, static_cast<uint64_t>(blockIdx.x) * blockDim.x, leaves, parent, n,
                      tree_folds, head, cap, ffa_seg, g, rc, rs, sp, thr_keep, scores, folds_out,
                      minmax);
}

// ---- end of a run: ascend and report --------------------------------------

// Ascend resolve of one leaf for one segment (poly_taylor_ascend_resolve_
// {accel,jerk}_batch, lib/taylor.cpp:693-813; poly_chebyshev_ascend_resolve_
// {accel,jerk}_batch, lib/chebyshev.cpp:1181-1312): the leaf carried from the
// middle coordinate (t_mid, scale s_mid) to the segment centre, in the
// reference's association.
__device__ __forceinline__ void ascend_resolve_leaf(const double* lf, const LeafGeom& g,
                                                    double dt, double inv_ts, uint32_t* pidx,
                                                    float* phase) {
    double a_new, v_new, d_new, f0;
    if (g.basis == 0 && g.np == 2) {
        const double half_dt2 = 0.5 * (dt * dt);
        const double a_cur = lf[0], v_cur = lf[2], d_cur = lf[4];
        f0 = lf[6];
        a_new = a_cur;
        v_new = v_cur + (a_cur * dt);
        d_new = d_cur + (v_cur * dt) + (a_cur * half_dt2);
    } else if (g.basis == 0) {
        const double half_dt2 = 0.5 * (dt * dt);
        const double sixth_dt3 = (half_dt2 * dt) / 3.0;
        const double j_cur = lf[0], a_cur = lf[2], v_cur = lf[4], d_cur = lf[6];
        f0 = lf[8];
        a_new = a_cur + (j_cur * dt);
        v_new = v_cur + (a_cur * dt) + (j_cur * half_dt2);
        d_new = d_cur + (v_cur * dt) + (a_cur * half_dt2) + (j_cur * sixth_dt3);
    } else if (g.np == 2) {
        const double dt2 = dt * dt;
        const double inv_ts2 = inv_ts * inv_ts;
        const double alpha_2 = lf[0], alpha_1 = lf[2], alpha_0 = lf[4];
        f0 = lf[6];
        a_new = 4.0 * alpha_2 * inv_ts2;
        v_new = (alpha_1 * inv_ts) + (4.0 * alpha_2 * inv_ts2 * dt);
        d_new = (alpha_0 - alpha_2) + (alpha_1 * inv_ts * dt) + (2.0 * alpha_2 * inv_ts2 * dt2);
    } else {
        const double dt2 = dt * dt;
        const double dt3 = dt2 * dt;
        const double inv_ts2 = inv_ts * inv_ts;
        const double inv_ts3 = inv_ts2 * inv_ts;
        const double alpha_3 = lf[0], alpha_2 = lf[2], alpha_1 = lf[4], alpha_0 = lf[6];
        f0 = lf[8];
        a_new = (4.0 * alpha_2 * inv_ts2) + (24.0 * alpha_3 * dt * inv_ts3);
        v_new = ((alpha_1 - (3.0 * alpha_3)) * inv_ts) + (4.0 * alpha_2 * inv_ts2 * dt) +
                (12.0 * alpha_3 * inv_ts3 * dt2);
        d_new = (alpha_0 - alpha_2) + ((alpha_1 - (3.0 * alpha_3)) * dt * inv_ts) +
                (2.0 * alpha_2 * inv_ts2 * dt2) + (4.0 * alpha_3 * inv_ts3 * dt3);
    }
    const double f_new = f0 * (1.0 - (v_new * kInvCval));
    const double delay_rel = d_new * kInvCval;
    *phase = dev::phase_idx(dt, f0, g.nbins, delay_rel);
    const uint32_t ia = dev::nearest_idx(a_new, g.a_min, g.a_max, g.n_accel);
    const uint32_t jf = dev::nearest_idx(f_new, g.f_min, g.f_max, g.n_freq);
    *pidx = ia * g.n_freq + jf;
}

// ascend (PrunePoly{Taylor,Chebyshev}DPFuncts::ascend, lib/dynamic.cpp:
// 311-371,450-508): each survivor's fold rebuilt over the segments searched
// so far -- zero, then every segment in middle-out order rotated right by
// round(shift) and added (shift_add_ascend_linear_batch, lib/kernels.cpp:
// 1390-1416) -- and rescored; the previous score moves to scores_ep. A warp
// per survivor: lanes resolve 32 segments at a time in double precision and
// the warp adds the segments' rows in order, each lane owning the bins
// j = lane mod 32 of a shared-memory accumulator. Then a thread per survivor
// scores its normalised row (the leaf step's scorer).
template <int NW, int NB>
__global__ void ascend_kernel(const double* __restrict__ leaves, uint64_t head, uint64_t cap,
                              uint64_t n, const float* __restrict__ ffa, uint64_t ncoords,
                              const uint32_t* __restrict__ seg_order, uint32_t nsegs, double tseg,
                              double t_mid, double inv_ts_mid, LeafGeom g, uint32_t rs,
                              ScoreParams sp, float* __restrict__ folds, float* __restrict__ scores,
                              float* __restrict__ scores_ep) {
    extern __shared__ float rows[];
    const uint32_t T = blockDim.x;
    const uint32_t nb = g.nbins;
    const uint32_t warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    float* acc = rows + static_cast<size_t>(T) * rs + static_cast<size_t>(warp) * 2 * nb;
    const uint64_t c0 = static_cast<uint64_t>(blockIdx.x) * T;
    const uint32_t nhere = static_cast<uint32_t>((n - c0) < T ? (n - c0) : T);
    for (uint32_t p = warp; p < nhere; p += T / kWarp) {
        const uint64_t phys = (head + c0 + p) % cap;
        const double* lf = leaves + phys * g.ls;
        // each lane touches only its own bins (E row j and V row nb + j)
        for (uint32_t j = lane; j < nb; j += kWarp) {
            acc[j] = 0.0f;
            acc[nb + j] = 0.0f;
        }
        for (uint32_t base = 0; base < nsegs; base += kWarp) {
            uint32_t my_pidx = 0, my_shift = 0;
            if (base + lane < nsegs) {
                const double t_seg = (static_cast<double>(seg_order[base + lane]) + 0.5) * tseg;
                float ph;
                ascend_resolve_leaf(lf, g, t_seg - t_mid, inv_ts_mid, &my_pidx, &ph);
                my_shift = dev::shift_bins(ph, nb);
            }
            const uint32_t cnt = (nsegs - base) < kWarp ? (nsegs - base) : kWarp;
            for (uint32_t q = 0; q < cnt; ++q) {
                const uint32_t pidx = __shfl_sync(0xffffffffu, my_pidx, q);
                const uint32_t sh = __shfl_sync(0xffffffffu, my_shift, q);
                const float* src =
                    ffa + (static_cast<uint64_t>(seg_order[base + q]) * ncoords + pidx) * 2 * nb;
                for (uint32_t j = lane; j < nb; j += kWarp) {
                    const uint32_t jh = j >= sh ? j - sh : j + nb - sh;
                    acc[j] = __fadd_rn(acc[j], __ldg(src + jh));
                    acc[nb + j] = __fadd_rn(acc[nb + j], __ldg(src + nb + jh));
                }
            }
        }
        float* o = folds + phys * 2 * nb;
        float* dst = rows + static_cast<size_t>(p) * rs;
        for (uint32_t j = lane; j < nb; j += kWarp) {
            o[j] = acc[j];
            o[nb + j] = acc[nb + j];
            dst[j] = sc::normalise(acc[j], acc[nb + j]);
        }
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x < nhere) {
        const uint64_t phys = (head + c0 + threadIdx.x) % cap;
        float score;
        sc::score_row_any<NB, NW>(rows + static_cast<size_t>(threadIdx.x) * rs, nb, 1.0f, sp,
                                  LK_SCORE_MAX, &score);
        scores_ep[phys] = scores[phys];
        scores[phys] = score;
    }
}

// report (PrunePoly{Taylor,Chebyshev}DPFuncts::report, lib/dynamic.cpp:
// 373-379,510-519): Chebyshev leaves to Taylor at the middle coordinate, then
// poly_taylor_report_batch (lib/taylor.cpp:1529-1564), the gauge transform to
// the observer frame with first-order error propagation.
__global__ void report_kernel(double* __restrict__ leaves, uint64_t head, uint64_t cap, uint64_t n,
                              uint32_t np, uint32_t basis, double ts_mid) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    double* lf = leaves + ((head + i) % cap) * ((np + 2) * 2);
    if (basis == 1) {
        cheby_to_taylor_leaf(lf, np, ts_mid);
    }
    const double v_final = lf[(np - 1) * 2 + 0];
    const double dv_final = lf[(np - 1) * 2 + 1];
    const double f0_batch = lf[(np + 1) * 2 + 0];
    const double s_factor = 1.0 - (v_final * kInvCval);
    for (uint32_t j = 0; j + 1 < np; ++j) {
        const double val = lf[j * 2 + 0];
        const double err = lf[j * 2 + 1];
        lf[j * 2 + 0] = val / s_factor;
        lf[j * 2 + 1] = sqrt(((err / s_factor) * (err / s_factor)) +
                             ((val * kInvCval / (s_factor * s_factor)) *
                              (val * kInvCval / (s_factor * s_factor)) * (dv_final * dv_final)));
    }
    lf[(np - 1) * 2 + 0] = f0_batch * s_factor;
    lf[(np - 1) * 2 + 1] = f0_batch * dv_final * kInvCval;
}

// ---- threshold-dependent steps --------------------------------------------

// Children of batch b (child_starts[b0 + b] .. child_starts[b0 + b + 1]) with
// score >= *d_thr (score_and_filter's test, lib/score.cpp:250).
__global__ void batch_count_kernel(const float* __restrict__ scores,
                                   const uint64_t* __restrict__ child_starts, uint64_t b0,
                                   const float* __restrict__ d_thr,
                                   uint32_t* __restrict__ counts) {
    __shared__ uint32_t ws[32];
    const uint64_t b = b0 + blockIdx.x;
    const uint64_t lo = child_starts[b], hi = child_starts[b + 1];
    const float thr = *d_thr;
    uint32_t c = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        c += scores[i] >= thr ? 1u : 0u;
    }
    uint32_t total;
    blk::block_exclusive_scan(c, ws, &total);
    if (threadIdx.x == 0) {
        counts[blockIdx.x] = total;
    }
}

// Ordered compaction of (id, score) pairs. Source kind CHILDREN: ids are
// base + i and scores scores[base + i]; kind LIST: ids[i], scores[i].
// Predicate: score >= *d_thr (GT = false) or score > *d_thr (GT = true).
enum class Src { kChildren, kList };

template <Src S>
__device__ __forceinline__ void pc_load(const float* sc, const uint32_t* ids, uint64_t base,
                                        uint64_t i, float* s, uint32_t* id) {
    if constexpr (S == Src::kChildren) {
        *s = sc[base + i];
        *id = static_cast<uint32_t>(base + i);
    } else {
        *s = sc[i];
        *id = ids[i];
    }
}

template <bool GT>
__device__ __forceinline__ bool pc_pred(float s, float thr) {
    return GT ? (s > thr) : (s >= thr);
}

template <Src S, bool GT>
__global__ void pc_count_kernel(const float* __restrict__ sc, const uint32_t* __restrict__ ids,
                                uint64_t base, uint64_t n, const float* __restrict__ d_thr,
                                uint32_t* __restrict__ tile_counts) {
    __shared__ uint32_t ws[32];
    const float thr = *d_thr;
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    uint32_t c = 0;
#pragma unroll
    for (uint32_t q = 0; q < kScanPer; ++q) {
        if (t0 + q < n) {
            float s;
            uint32_t id;
            pc_load<S>(sc, ids, base, t0 + q, &s, &id);
            c += pc_pred<GT>(s, thr) ? 1u : 0u;
        }
    }
    uint32_t total;
    blk::block_exclusive_scan(c, ws, &total);
    if (threadIdx.x == 0) {
        tile_counts[blockIdx.x] = total;
    }
}

// Writes kept pairs at *d_base + rank, skipping ranks at or beyond
// limit - *d_base (the reference's min(pending, space_left)).
template <Src S, bool GT>
__global__ void pc_scatter_kernel(const float* __restrict__ sc, const uint32_t* __restrict__ ids,
                                  uint64_t base, uint64_t n, const float* __restrict__ d_thr,
                                  const uint64_t* __restrict__ tile_offs,
                                  const uint64_t* __restrict__ d_base, uint64_t limit,
                                  uint32_t* __restrict__ out_ids, float* __restrict__ out_sc) {
    __shared__ uint32_t ws[32];
    const float thr = *d_thr;
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * kScanTile + threadIdx.x * kScanPer;
    float s[kScanPer];
    uint32_t id[kScanPer];
    uint32_t c = 0;
#pragma unroll
    for (uint32_t q = 0; q < kScanPer; ++q) {
        s[q] = 0.0f;
        id[q] = 0;
        if (t0 + q < n) {
            pc_load<S>(sc, ids, base, t0 + q, &s[q], &id[q]);
        }
        c += (t0 + q < n && pc_pred<GT>(s[q], thr)) ? 1u : 0u;
    }
    uint64_t pos = *d_base + tile_offs[blockIdx.x] + blk::block_exclusive_scan(c, ws, nullptr);
#pragma unroll
    for (uint32_t q = 0; q < kScanPer; ++q) {
        if (t0 + q < n && pc_pred<GT>(s[q], thr)) {
            if (pos < limit) {
                out_ids[pos] = id[q];
                out_sc[pos] = s[q];
            }
            ++pos;
        }
    }
}

// *d_size_out = min(*d_base + *d_total, limit).
__global__ void pc_finish_kernel(const uint64_t* d_base, const uint64_t* d_total, uint64_t limit,
                                 uint64_t* d_size_out) {
    const uint64_t v = *d_base + *d_total;
    *d_size_out = v < limit ? v : limit;
}

// WorldTree::get_prune_threshold (lib/world_tree.cpp:570-618) on the
// candidates {list scores} U {children of one batch with score >= *d_thr}:
// N of them, K = size + space_left. The reference's two nth_element calls
// select fixed order statistics: with D sorted in descending order, the
// top-k value D[K-1] and the median value D[K-1-N/2] when N/2 <= K-1, else
// D[N-1-N/2+K]. Both are found exactly by an 8-bit MSD radix select over
// orderable keys (one block, four passes). The new threshold
// max(current, nextafter(topk), nextafter(median)) replaces *d_thr.
// The body, for one block of any size: returns the new threshold (to every
// thread) for the current threshold thr.
__device__ float select_threshold_block(const float* __restrict__ list_sc, uint64_t size,
                                        const float* __restrict__ scores, uint64_t cb0,
                                        uint64_t cb1, uint64_t N, uint64_t r_topk,
                                        uint64_t r_med, float thr, float* d_debug) {
    __shared__ uint32_t hist[2][256];
    __shared__ uint32_t prefix[2];
    __shared__ uint64_t q[2];
    __shared__ float s_eff;
    if (threadIdx.x < 2) {
        prefix[threadIdx.x] = 0;
        // ascending rank of the wanted descending rank
        q[threadIdx.x] = N - 1 - (threadIdx.x == 0 ? r_topk : r_med);
    }
    for (int pass = 0; pass < 4; ++pass) {
        const uint32_t shift = 24u - 8u * static_cast<uint32_t>(pass);
        const uint32_t hmask = pass == 0 ? 0u : (0xffffffffu << (shift + 8u));
        for (uint32_t i = threadIdx.x; i < 512; i += blockDim.x) {
            hist[i / 256][i % 256] = 0;
        }
        __syncthreads();
        const uint32_t p0 = prefix[0] & hmask, p1 = prefix[1] & hmask;
        for (uint64_t i = threadIdx.x; i < size; i += blockDim.x) {
            const uint32_t k = fkey(list_sc[i]);
            const uint32_t d = (k >> shift) & 0xffu;
            if ((k & hmask) == p0) atomicAdd(&hist[0][d], 1u);
            if ((k & hmask) == p1) atomicAdd(&hist[1][d], 1u);
        }
        for (uint64_t c = cb0 + threadIdx.x; c < cb1; c += blockDim.x) {
            const float s = scores[c];
            if (s >= thr) {
                const uint32_t k = fkey(s);
                const uint32_t d = (k >> shift) & 0xffu;
                if ((k & hmask) == p0) atomicAdd(&hist[0][d], 1u);
                if ((k & hmask) == p1) atomicAdd(&hist[1][d], 1u);
            }
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            const uint32_t r = threadIdx.x;
            uint64_t acc = 0;
            uint32_t d = 0;
            for (; d < 255; ++d) {
                if (q[r] < acc + hist[r][d]) {
                    break;
                }
                acc += hist[r][d];
            }
            q[r] -= acc;
            prefix[r] |= d << shift;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const float topk = nextafterf(fkey_inv(prefix[0]), FLT_MAX);
        const float med = nextafterf(fkey_inv(prefix[1]), FLT_MAX);
        float eff = thr;
        eff = (eff < topk) ? topk : eff;
        eff = (eff < med) ? med : eff;
        s_eff = eff;
        if (d_debug != nullptr) {
            d_debug[0] = fkey_inv(prefix[0]);
            d_debug[1] = fkey_inv(prefix[1]);
        }
    }
    __syncthreads();
    const float eff = s_eff;
    __syncthreads();  // s_eff, hist and prefix are free for the next call
    (void)N;
    return eff;
}

__global__ void select_threshold_kernel(const float* __restrict__ list_sc, uint64_t size,
                                        const float* __restrict__ scores, uint64_t cb0,
                                        uint64_t cb1, uint64_t N, uint64_t r_topk,
                                        uint64_t r_med, float* d_thr, float* d_debug) {
    const float eff = select_threshold_block(list_sc, size, scores, cb0, cb1, N, r_topk, r_med,
                                             *d_thr, d_debug);
    if (threadIdx.x == 0) {
        *d_thr = eff;
    }
}

// Level end: transform (poly_taylor_transform_{accel,jerk}_batch,
// lib/taylor.cpp:881-1005) and gather the survivors into the tree at
// physical slots (write_start + i) mod cap. One warp per survivor.
struct TransformConsts {
    double dt, half_dt2, sixth_dt3, dt2;
    int conservative;
    // Chebyshev (lib/chebyshev.cpp:316-409): p = s_next / s_cur, q = dt / s_cur
    int basis;
    double p, q, p2, q2, pq, p3;
};

// poly_chebyshev_transform_{accel,jerk}_batch: values through the
// re-centring matrix, errors times its diagonal (non-conservative).
__device__ __forceinline__ void cheby_transform_leaf(const double* in, double* o, uint32_t np,
                                                     const TransformConsts& tc) {
    const double p = tc.p, q = tc.q, p2 = tc.p2, q2 = tc.q2;
    for (uint32_t k = 0; k < (np + 2) * 2; ++k) {
        o[k] = in[k];
    }
    if (np == 2) {
        const double a2v = in[0], a2e = in[1], a1v = in[2], a1e = in[3], a0v = in[4];
        o[0] = p2 * a2v;
        o[2] = (p * a1v) + (4.0 * tc.pq * a2v);
        o[4] = a0v + (q * a1v) + ((p2 + (2.0 * q2) - 1.0) * a2v);
        o[1] = p2 * a2e;
        o[3] = p * a1e;
    } else {
        const double p3 = tc.p3;
        const double a3v = in[0], a3e = in[1], a2v = in[2], a2e = in[3], a1v = in[4],
                     a1e = in[5], a0v = in[6];
        o[0] = p3 * a3v;
        o[2] = (6.0 * p2 * q * a3v) + (p2 * a2v);
        o[4] = (3.0 * p * (p2 + (4.0 * q2) - 1.0) * a3v) + (4.0 * p * q * a2v) + (p * a1v);
        o[6] = (q * ((6.0 * p2) + (4.0 * q2) - 3.0) * a3v) + ((p2 + (2.0 * q2) - 1.0) * a2v) +
               (q * a1v) + a0v;
        o[1] = p3 * a3e;
        o[3] = p2 * a2e;
        o[5] = p * a1e;
    }
}

__device__ __forceinline__ void transform_leaf(const double* in, double* o, uint32_t np,
                                               const TransformConsts& tc) {
    if (tc.basis == 1) {
        cheby_transform_leaf(in, o, np, tc);
        return;
    }
    const double dt = tc.dt;
    if (np == 2) {
        const double d2v = in[0], d2e = in[1], d1v = in[2], d1e = in[3], d0v = in[4],
                     d0e = in[5];
        const double d1v_j = d1v + (d2v * dt);
        const double d0v_j = d0v + (d1v * dt) + (d2v * tc.half_dt2);
        const double d1e_j =
            tc.conservative ? __dsqrt_rn((d1e * d1e) + (d2e * d2e * dt * dt)) : d1e;
        o[0] = d2v;
        o[1] = d2e;
        o[2] = d1v_j;
        o[3] = d1e_j;
        o[4] = d0v_j;
        o[5] = d0e;
        o[6] = in[6];
        o[7] = in[7];
    } else {
        const double d3v = in[0], d3e = in[1], d2v = in[2], d2e = in[3], d1v = in[4],
                     d1e = in[5], d0v = in[6], d0e = in[7];
        const double d2v_j = d2v + (d3v * dt);
        const double d1v_j = d1v + (d2v * dt) + (d3v * tc.half_dt2);
        const double d0v_j = d0v + (d1v * dt) + (d2v * tc.half_dt2) + (d3v * tc.sixth_dt3);
        double d2e_j = d2e, d1e_j = d1e;
        if (tc.conservative) {
            d2e_j = __dsqrt_rn((d2e * d2e) + (d3e * d3e * tc.dt2));
            d1e_j = __dsqrt_rn((d1e * d1e) + (d2e * d2e * tc.dt2) +
                               (d3e * d3e * tc.half_dt2 * tc.half_dt2));
        }
        o[0] = d3v;
        o[1] = d3e;
        o[2] = d2v_j;
        o[3] = d2e_j;
        o[4] = d1v_j;
        o[5] = d1e_j;
        o[6] = d0v_j;
        o[7] = d0e;
        o[8] = in[8];
        o[9] = in[9];
    }
}

// Survivor w of the write list (one warp): transformed leaf, fold and score
// into physical slot (write_start + w) mod cap of the other tree buffer.
__device__ __forceinline__ void gather_one(uint64_t w, uint32_t lane, const uint32_t* __restrict__ list_ids,
                                           const float* __restrict__ list_sc,
                                           const double* __restrict__ leaves,
                                           const float* __restrict__ folds, uint64_t write_start,
                                           uint64_t cap, uint32_t np, uint32_t nbins,
                                           const TransformConsts& tc, double* __restrict__ t_leaves,
                                           float* __restrict__ t_folds, float* __restrict__ t_scores) {
    const uint64_t c = list_ids[w];
    const uint64_t ph = (write_start + w) % cap;
    const uint32_t ls = (np + 2) * 2;
    if (lane == 0) {
        transform_leaf(leaves + c * ls, t_leaves + ph * ls, np, tc);
        t_scores[ph] = list_sc[w];
    }
    const float* src = folds + c * 2 * nbins;
    float* dst = t_folds + ph * 2 * nbins;
    for (uint32_t j = lane; j < 2 * nbins; j += kWarp) {
        dst[j] = src[j];
    }
}

__global__ void gather_kernel(const uint32_t* __restrict__ list_ids,
                              const float* __restrict__ list_sc, uint64_t size,
                              const double* __restrict__ leaves, const float* __restrict__ folds,
                              uint64_t write_start, uint64_t cap, uint32_t np, uint32_t nbins,
                              TransformConsts tc, double* __restrict__ t_leaves,
                              float* __restrict__ t_folds, float* __restrict__ t_scores) {
    const uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp;
    if (w >= size) {
        return;
    }
    gather_one(w, threadIdx.x % kWarp, list_ids, list_sc, leaves, folds, write_start, cap, np, nbins,
               tc, t_leaves, t_folds, t_scores);
}

// In-place transform of leaves named by indices (the standalone entry
// point); an index at or beyond n_leaves is skipped and flagged.
__global__ void transform_kernel(double* __restrict__ leaves, uint64_t n_leaves,
                                 const uint32_t* __restrict__ idx, uint64_t n, uint32_t np,
                                 TransformConsts tc, uint32_t* status) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    if (idx[i] >= n_leaves) {
        atomicOr(status, dev::kStatusBadTable);
        return;
    }
    double* lf = leaves + static_cast<uint64_t>(idx[i]) * (np + 2) * 2;
    double tmp[10];
    transform_leaf(lf, tmp, np, tc);
    for (uint32_t q = 0; q < (np + 2) * 2; ++q) {
        lf[q] = tmp[q];
    }
}

// Chebyshev branch, first step (lib/chebyshev.cpp:516-522, 660-666): the
// level's parents, at physical slots (head + i) mod cap, re-centred in place
// from coord_prev to coord_cur.
__global__ void parent_transform_kernel(double* __restrict__ tree_leaves, uint64_t head,
                                        uint64_t cap, uint64_t n, uint32_t np,
                                        TransformConsts tc) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) {
        return;
    }
    double* lf = tree_leaves + ((head + i) % cap) * (np + 2) * 2;
    double tmp[10];
    transform_leaf(lf, tmp, np, tc);
    for (uint32_t q = 0; q < (np + 2) * 2; ++q) {
        lf[q] = tmp[q];
    }
}

// ---- persistent tail of a run -----------------------------------------------
//
// Once the tree is small, a level's kernels are short and the level is bound
// by launches and by the two host round trips of its batch replay. The tail
// kernel runs the remaining levels in ONE cooperative launch (one block per
// SM): the same steps and the same device functions as the level-by-level
// path, separated by grid barriers, with the batch replay (sizes, space left,
// batch boundaries at the buffer's wrap, overload steps) done by block 0 on
// the device. It hands the run back to the host, before changing anything,
// when a level has more parents or children than its buffers hold.

constexpr uint32_t kTailBatches = 64;    // batches of one level (wrap splits included)
constexpr uint64_t kTailParents = 16384;  // largest level (parents) the tail runs
constexpr uint64_t kTailChildren = 1 << 17;  // most children of one tail level
// Block 0 alone runs a tree's levels once a level has at most this many
// parents and the level before at most this many children; a level with more
// than kTailSoloMaxParents parents then goes back to the host.
constexpr uint64_t kTailSoloParents = 64;
constexpr uint64_t kTailSoloChildren = 256;
constexpr uint64_t kTailSoloMaxParents = 1024;
constexpr uint32_t kTailExitNone = 0;
constexpr uint32_t kTailExitDone = 1;    // every level run, or the tree emptied
constexpr uint32_t kTailExitHandBack = 2;  // level `level` too large: host continues
constexpr uint32_t kTailExitError = 3;   // status bits / reason set; the host fails
constexpr uint32_t kTailReasonBatch = 1; // a batch's children exceed batch_size * branch_max
constexpr uint32_t kTailReasonBig = 2;   // a level's children exceed 2^32 - 1

// One level's constants (host-computed, as the level-by-level path does).
struct TailLevel {
    const float* seg;      // FFA segment of the level
    float threshold;
    double dt;             // current coordinate's scale (branching)
    ResolveConsts rc;
    TransformConsts tc;    // survivors to the next coordinate
    TransformConsts pt;    // Chebyshev: parents re-centred first
};

// Device-resident state of the tail (zeroed barrier words, the tree entering
// the first level; the rest is scratch written by block 0).
struct TailCtl {
    uint64_t head, size;
    uint32_t cur, level, exit, reason;
    uint32_t status;
    uint32_t bar_count, bar_gen;
    uint32_t li, nbat;
    float thr;
    uint64_t n_par, n_child, write_start;
    uint64_t bstart[kTailBatches + 1], bsize[kTailBatches], cstart[kTailBatches + 1];
    uint32_t active;       // 0: all the tree's blocks; 1: block 0 alone (small levels)
};

struct TailArgs {
    double* tleaves[2];
    float* tfolds[2];
    float* tscores[2];
    uint32_t* lids[2];
    float* lsc[2];
    double* cleaves;
    uint32_t* cparent;
    float* cscores;
    float* cfolds;
    double* tp;            // re-centred parents (Chebyshev)
    uint32_t* counts;
    uint64_t* offsets;
    const TailLevel* lconst;  // indexed by level
    TailCtl* ctl;
    uint64_t* stats;       // per level: parents, children, survivors
    uint32_t* level_mm;    // per level: orderable min / max score keys
    uint64_t cap, batch, branch_max, max_parents, max_children;
    uint32_t last_level, rs;
    LeafGeom geom;
    ScoreParams sp;
};

// Barrier of one tree's nblocks blocks in a cooperative launch (all blocks
// resident), bounded like every device wait here: false (and the status bit
// set) when it gave up.
__device__ bool tail_barrier(TailCtl* ctl, uint32_t nblocks) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile uint32_t* gen = &ctl->bar_gen;
        const uint32_t g0 = *gen;
        __threadfence();
        if (atomicAdd(&ctl->bar_count, 1u) == nblocks - 1) {
            atomicExch(&ctl->bar_count, 0u);
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            const uint64_t t0 = ptx::globaltimer_ns();
            uint32_t it = 0;
            while (*gen == g0) {
                ++it;
                if (((it & 255u) == 0 && ptx::globaltimer_ns() - t0 > ptx::kWaitLimitNs) ||
                    it >= (1u << 26)) {
                    atomicOr(&ctl->status, dev::kStatusWaitTimeout);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Ordered compaction by one block: items [0, n) kept by keep(i) are written
// as (id(i), score(i)) at out[pos + rank] while pos + rank < limit; returns
// the number kept. Thread t takes a contiguous run of the items.
template <class Keep, class Id, class Score>
__device__ uint64_t block_append(uint64_t n, Keep keep, Id id, Score score, uint32_t* out_ids,
                                 float* out_sc, uint64_t pos, uint64_t limit) {
    __shared__ uint32_t ws[32];
    const uint64_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint64_t i0 = threadIdx.x * per;
    const uint64_t i1 = min(n, i0 + per);
    uint32_t c = 0;
    for (uint64_t i = i0; i < i1; ++i) {
        c += keep(i) ? 1u : 0u;
    }
    uint32_t total;
    uint64_t o = pos + blk::block_exclusive_scan(c, ws, &total);
    for (uint64_t i = i0; i < i1; ++i) {
        if (keep(i)) {
            if (o < limit) {
                out_ids[o] = id(i);
                out_sc[o] = score(i);
            }
            ++o;
        }
    }
    __syncthreads();  // ws is reused by the next scan
    return total;
}

template <int NW, int NB>
__global__ void __launch_bounds__(128) prune_tail_kernel(const TailArgs* __restrict__ trees, uint32_t bpt) {
    extern __shared__ float rows[];
    // blocks [t * bpt, (t + 1) * bpt) run tree t; lb is the block's index there
    const uint32_t lb = blockIdx.x % bpt;
    const TailArgs& a = trees[blockIdx.x / bpt];
    TailCtl* ctl = a.ctl;
    // values other blocks wrote before a barrier are read through vc
    volatile TailCtl* vc = a.ctl;
    // blocks taking part in the tree's barriers (all, until the tree is small)
    uint32_t nblk = vc->active != 0 ? vc->active : bpt;
    const LeafGeom& g = a.geom;
    const uint32_t np = g.np, ls = g.ls, nb = g.nbins;
    const uint64_t cap = a.cap;
    for (;;) {
        // 0. the level's set-up (block 0, thread 0): batches as get_leaves_span
        if (lb == 0 && threadIdx.x == 0) {
            const uint32_t lv = ctl->level;
            const uint64_t n_par = ctl->size;
            if (lv > a.last_level || n_par == 0) {
                ctl->exit = kTailExitDone;
            } else if (n_par > a.max_parents) {
                ctl->exit = kTailExitHandBack;
            } else {
                const uint64_t bmin = a.batch < n_par ? a.batch : n_par;
                const uint64_t bs = bmin > 0 ? bmin : 1;
                uint32_t nbat = 0;
                uint64_t done = 0;
                while (done < n_par && nbat < kTailBatches) {
                    const uint64_t want = min(bs, n_par - done);
                    const uint64_t phys = (ctl->head + done) % cap;
                    const uint64_t take = min(want, cap - phys);
                    ctl->bstart[nbat] = done;
                    ctl->bsize[nbat] = take;
                    done += take;
                    ++nbat;
                }
                if (ctl->active == 0 && n_par <= kTailSoloParents && ctl->n_child <= kTailSoloChildren) {
                    // a small tree: the other blocks leave, block 0 runs the
                    // remaining levels alone (block barriers, no grid waits)
                    ctl->active = 1;
                }
                if (done < n_par || (ctl->active == 1 && n_par > kTailSoloMaxParents)) {
                    ctl->exit = kTailExitHandBack;
                } else {
                    ctl->bstart[nbat] = n_par;
                    ctl->nbat = nbat;
                    ctl->n_par = n_par;
                    ctl->write_start = (ctl->head + n_par) % cap;
                    ctl->thr = a.lconst[lv].threshold;
                    a.level_mm[2 * lv] = 0xffffffffu;
                    a.level_mm[2 * lv + 1] = 0u;
                }
            }
        }
        if (!tail_barrier(ctl, nblk) || vc->exit != kTailExitNone) {
            return;
        }
        nblk = vc->active != 0 ? vc->active : bpt;
        if (lb >= nblk) {
            return;  // the level runs on fewer blocks from here on
        }
        const uint32_t lv = vc->level;
        const TailLevel& L = a.lconst[lv];
        const uint64_t n_par = vc->n_par, head = vc->head;
        const int cur = static_cast<int>(vc->cur);
        const double* tree = a.tleaves[cur];
        const uint64_t gtid = static_cast<uint64_t>(lb) * blockDim.x + threadIdx.x;
        const uint64_t gthreads = static_cast<uint64_t>(nblk) * blockDim.x;

        // 1. branch counts (Chebyshev: parents re-centred into tp, the tree
        //    is not written, so a hand-back leaves it as it was)
        for (uint64_t i = gtid; i < n_par; i += gthreads) {
            const double* lf = tree + ((head + i) % cap) * ls;
            if (g.basis == 1) {
                double* t = a.tp + i * ls;
                double tmp[10];
                transform_leaf(lf, tmp, np, L.pt);
                for (uint32_t q = 0; q < ls; ++q) {
                    t[q] = tmp[q];
                }
                lf = t;
            }
            ParamBranch pb[3];
            branch_params(lf, L.dt, g, pb, &ctl->status);
            uint64_t prod = 1;
            for (uint32_t k = 0; k < np; ++k) {
                prod *= pb[k].count;
            }
            if (prod > 0xffffffffull) {
                atomicOr(&ctl->status, kStatusBranchCount);
                prod = 1;
            }
            a.counts[i] = static_cast<uint32_t>(prod);
        }
        if (!tail_barrier(ctl, nblk)) {
            return;
        }
        // 2. offsets, batch child ranges, checks (block 0)
        if (lb == 0) {
            __shared__ uint32_t ws[32];
            const uint64_t per = (n_par + blockDim.x - 1) / blockDim.x;
            const uint64_t i0 = threadIdx.x * per, i1 = min(n_par, i0 + per);
            uint64_t c = 0;
            for (uint64_t i = i0; i < i1; ++i) {
                c += a.counts[i];
            }
            // the exact total first: below 2^32 the 32-bit scan is exact too
            // (a larger total ends the tail with an error before any use)
            __shared__ unsigned long long s_total;
            if (threadIdx.x == 0) {
                s_total = 0;
            }
            __syncthreads();
            atomicAdd(&s_total, static_cast<unsigned long long>(c));
            uint32_t tot32;
            uint64_t o = blk::block_exclusive_scan(static_cast<uint32_t>(c), ws, &tot32);
            __syncthreads();
            for (uint64_t i = i0; i < i1; ++i) {
                a.offsets[i] = o;
                o += a.counts[i];
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const uint64_t n_child = s_total;
                const uint32_t nbat = ctl->nbat;
                ctl->n_child = n_child;
                for (uint32_t b = 0; b <= nbat; ++b) {
                    ctl->cstart[b] = ctl->bstart[b] < n_par ? a.offsets[ctl->bstart[b]] : n_child;
                }
                const uint32_t st = ctl->status;
                if (st & (kStatusBranchMax | kStatusZeroStep | kStatusBranchCount)) {
                    ctl->exit = kTailExitError;
                } else if (n_child >= (1ull << 32)) {
                    ctl->exit = kTailExitError;
                    ctl->reason = kTailReasonBig;
                } else {
                    for (uint32_t b = 0; b < nbat; ++b) {
                        if (ctl->cstart[b + 1] - ctl->cstart[b] > a.batch * a.branch_max) {
                            ctl->exit = kTailExitError;
                            ctl->reason = kTailReasonBatch;
                        }
                    }
                    if (ctl->exit == kTailExitNone && n_child > a.max_children) {
                        ctl->exit = kTailExitHandBack;
                    }
                }
            }
        }
        if (!tail_barrier(ctl, nblk) || vc->exit != kTailExitNone) {
            return;
        }
        const uint64_t n_child = vc->n_child;
        // 3. children's leaves (branch_emit_kernel's order)
        for (uint64_t i = gtid; i < n_par; i += gthreads) {
            const double* lf = g.basis == 1 ? a.tp + i * ls : tree + ((head + i) % cap) * ls;
            ParamBranch pb[3];
            branch_params(lf, L.dt, g, pb, &ctl->status);
            uint64_t o = a.offsets[i];
            const uint32_t c2 = np == 3 ? pb[2].count : 1;
            for (uint32_t x = 0; x < pb[0].count; ++x) {
                const double va = branch_value(pb[0], x);
                for (uint32_t y = 0; y < pb[1].count; ++y) {
                    const double vb = branch_value(pb[1], y);
                    for (uint32_t z = 0; z < c2; ++z) {
                        double* d = a.cleaves + o * ls;
                        d[0] = va;
                        d[1] = pb[0].dparam;
                        d[2] = vb;
                        d[3] = pb[1].dparam;
                        if (np == 3) {
                            d[4] = branch_value(pb[2], z);
                            d[5] = pb[2].dparam;
                        }
                        for (uint32_t q = 2 * np; q < ls; ++q) {
                            d[q] = lf[q];
                        }
                        a.cparent[o] = static_cast<uint32_t>(i);
                        ++o;
                    }
                }
            }
        }
        if (!tail_barrier(ctl, nblk)) {
            return;
        }
        // 4. resolve, shift-add, score, kept folds (tiles of blockDim children)
        for (uint64_t c0 = static_cast<uint64_t>(lb) * blockDim.x; c0 < n_child;
             c0 += static_cast<uint64_t>(nblk) * blockDim.x) {
            leaf_tile<NW, NB>(rows, c0, a.cleaves, a.cparent, n_child, a.tfolds[cur], head, cap, L.seg,
                              g, L.rc, a.rs, a.sp, L.threshold, a.cscores, a.cfolds,
                              a.level_mm + 2 * lv);
            __syncthreads();
        }
        if (!tail_barrier(ctl, nblk)) {
            return;
        }
        // 5. filter + add in the reference's batch order (block 0)
        if (lb == 0) {
            const uint32_t nbat = vc->nbat;
            uint64_t size = 0, read_consumed = 0;
            int li = 0;
            float thr = L.threshold;
            const float* sc = a.cscores;
            for (uint32_t b = 0; b < nbat; ++b) {
                const uint64_t cb0 = vc->cstart[b], cb1 = vc->cstart[b + 1];
                __shared__ uint32_t ws[32];
                uint32_t cnt_local = 0;
                for (uint64_t i = cb0 + threadIdx.x; i < cb1; i += blockDim.x) {
                    cnt_local += sc[i] >= thr ? 1u : 0u;
                }
                uint32_t cnt;
                blk::block_exclusive_scan(cnt_local, ws, &cnt);
                __syncthreads();
                const uint64_t space = cap - ((n_par - read_consumed) + size);
                const uint64_t nb_c = cb1 - cb0;
                auto child_id = [&](uint64_t i) { return static_cast<uint32_t>(cb0 + i); };
                auto child_sc = [&](uint64_t i) { return sc[cb0 + i]; };
                if (cnt <= space) {
                    const float t = thr;
                    size += block_append(nb_c, [&](uint64_t i) { return sc[cb0 + i] >= t; }, child_id, child_sc,
                                         a.lids[li], a.lsc[li], size, cap);
                } else {
                    // overload (lib/world_tree.cpp:386-421)
                    const uint64_t K = size + space;
                    const uint64_t N = size + cnt;
                    const uint64_t m = N / 2;
                    const uint64_t r_med = (m <= K - 1) ? (K - 1 - m) : (N - 1 - m + K);
                    thr = select_threshold_block(a.lsc[li], size, sc, cb0, cb1, N, K - 1, r_med, thr,
                                                 nullptr);
                    const float t = thr;
                    const uint32_t* lid = a.lids[li];
                    const float* lsc = a.lsc[li];
                    const uint64_t kept = block_append(
                        size, [&](uint64_t i) { return lsc[i] > t; }, [&](uint64_t i) { return lid[i]; },
                        [&](uint64_t i) { return lsc[i]; }, a.lids[1 - li], a.lsc[1 - li], 0, cap);
                    const uint64_t added = block_append(
                        nb_c, [&](uint64_t i) { return sc[cb0 + i] >= t; }, child_id, child_sc,
                        a.lids[1 - li], a.lsc[1 - li], kept, K);
                    size = min(kept + added, K);
                    li = 1 - li;
                }
                read_consumed += vc->bsize[b];
            }
            if (threadIdx.x == 0) {
                ctl->li = static_cast<uint32_t>(li);
                ctl->size = size;  // survivors (the next level's parents)
                ctl->thr = thr;
            }
        }
        if (!tail_barrier(ctl, nblk)) {
            return;
        }
        // 6. survivors transformed and gathered into the other tree buffer
        {
            const uint64_t size = vc->size;
            const int li = static_cast<int>(vc->li);
            const uint64_t ws0 = vc->write_start;
            const int nxt = 1 - cur;
            const uint64_t gw = gtid / kWarp, nwarps = gthreads / kWarp;
            for (uint64_t w = gw; w < size; w += nwarps) {
                gather_one(w, threadIdx.x % kWarp, a.lids[li], a.lsc[li], a.cleaves, a.cfolds, ws0, cap, np,
                           nb, L.tc, a.tleaves[nxt], a.tfolds[nxt], a.tscores[nxt]);
            }
        }
        if (!tail_barrier(ctl, nblk)) {
            return;
        }
        // 7. the level's end (finalize_in_place_update) and its statistics
        if (lb == 0 && threadIdx.x == 0) {
            const uint64_t size = ctl->size;
            a.stats[3 * lv] = n_par;
            a.stats[3 * lv + 1] = n_child;
            a.stats[3 * lv + 2] = size;
            ctl->head = ctl->write_start;
            if (size > 0) {
                ctl->cur = 1u - ctl->cur;
            }
            ctl->level = lv + 1;
        }
        // the next level's set-up waits at its first barrier
    }
}

// Launch shape of the tail kernel: blockDim = the leaf kernel's tile, its
// rows and per-child words in dynamic shared memory.
uint32_t tail_threads(uint32_t rs) { return sc::profiles_per_block(rs + 4); }
size_t tail_smem(uint32_t rs) {
    const uint32_t T = tail_threads(rs);
    return static_cast<size_t>(T) * rs * sizeof(float) + 4 * T * sizeof(uint32_t);
}

template <class F>
void with_tail_kernel(const ScoreParams& sp, uint32_t nbins, F&& f) {
    sc::dispatch_nw_nb(sp.nwidths, nbins, [&](auto nw, auto nbc) {
        f(prune_tail_kernel<decltype(nw)::value, decltype(nbc)::value>);
    });
}

// Tail blocks that fit one SM together.
uint32_t tail_blocks_per_sm(const ScoreParams& sp, uint32_t nbins, uint32_t rs) {
    int per_sm = 0;
    with_tail_kernel(sp, nbins, [&](auto kern) {
        sc::set_smem(kern, tail_smem(rs));
        LK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, static_cast<int>(tail_threads(rs)),
                                                              tail_smem(rs)));
    });
    require(per_sm >= 1, "pruning tail: one block per SM does not fit");
    return static_cast<uint32_t>(per_sm);
}

// ntrees trees (TailArgs on the device), bpt blocks each, all resident: a
// cooperative launch, since each tree's blocks wait on one another at its
// barriers.
void launch_tails(const TailArgs* d_args, uint32_t ntrees, uint32_t bpt, const ScoreParams& sp,
                  uint32_t nbins, uint32_t rs, cudaStream_t s) {
    int dev = 0, nsm = 148;
    LK_CUDA(cudaGetDevice(&dev));
    LK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t per_sm = tail_blocks_per_sm(sp, nbins, rs);
    require(static_cast<uint64_t>(ntrees) * bpt <= static_cast<uint64_t>(per_sm) * static_cast<uint32_t>(nsm),
            "pruning tail: more blocks than the device holds at once");
    with_tail_kernel(sp, nbins, [&](auto kern) {
        const TailArgs* trees = d_args;
        void* args[] = {&trees, &bpt};
        LK_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), dim3(ntrees * bpt),
                                            dim3(tail_threads(rs)), args, tail_smem(rs), s));
    });
    LK_CUDA(cudaGetLastError());
}

__global__ void set_u64_kernel(uint64_t* p, uint64_t v) { *p = v; }
__global__ void init_minmax_kernel(uint32_t* mm) {
    mm[0] = 0xffffffffu;
    mm[1] = 0u;
}
// A level's starting state in one launch: its threshold, an empty write
// list and its score min / max slot.
__global__ void level_init_kernel(float* thr, float v, uint64_t* size, uint32_t* mm) {
    *thr = v;
    *size = 0;
    mm[0] = 0xffffffffu;
    mm[1] = 0u;
}

}  // namespace

namespace {

// misc buffer layout (bytes)
constexpr size_t kMiscThr = 0;      // float: current threshold
constexpr size_t kMiscZero = 8;     // uint64: always 0
constexpr size_t kMiscSize0 = 16;   // uint64: size of list 0
constexpr size_t kMiscSize1 = 24;   // uint64: size of list 1
constexpr size_t kMiscTotal = 32;   // uint64: scan / compaction total
constexpr size_t kMiscMinMax = 40;  // uint32[2]: orderable min / max score keys
constexpr size_t kMiscDebug = 48;   // float[2]: selected order statistics
constexpr size_t kMiscBytes = 64;

float key_to_float(uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    std::memcpy(&f, &u, sizeof(f));
    return f;
}

// np.argsort(|arange(nseg) - ref|, kind="stable") (lib/loki/psr_utils.hpp:331-347).
std::vector<uint64_t> middle_out_order(uint64_t nseg, uint64_t ref) {
    std::vector<uint64_t> order;
    order.reserve(nseg);
    order.push_back(ref);
    for (uint64_t d = 1; order.size() < nseg; ++d) {
        if (d <= ref) {
            order.push_back(ref - d);
        }
        if (ref + d < nseg && order.size() < nseg) {
            order.push_back(ref + d);
        }
    }
    return order;
}

// MiddleOutScheme::get_coord / get_current_coord / get_segment_coord
// (lib/loki/psr_utils.hpp:378-448).
struct Coord {
    double ref, scale;
};
Coord mo_coord(const std::vector<uint64_t>& order, uint64_t level, double tseg) {
    uint64_t mn = order[0], mx = order[0];
    for (uint64_t i = 1; i <= level; ++i) {
        mn = std::min(mn, order[i]);
        mx = std::max(mx, order[i]);
    }
    const double min_val = static_cast<double>(mn);
    const double max_val = static_cast<double>(mx);
    const double ref_val = (min_val + max_val + 1.0) / 2.0;
    const double scale_val = ref_val - min_val;
    return {ref_val * tseg, scale_val * tseg};
}
Coord mo_current_coord(const std::vector<uint64_t>& order, uint64_t level, double tseg) {
    if (level == 0) {
        return mo_coord(order, 0, tseg);
    }
    return {mo_coord(order, level - 1, tseg).ref, mo_coord(order, level, tseg).scale};
}
Coord mo_segment_coord(const std::vector<uint64_t>& order, uint64_t level, double tseg) {
    const double idx = static_cast<double>(order[level]);
    return {(idx + 0.5) * tseg, 0.5 * tseg};
}

LeafGeom make_geom(const Plan& p, uint64_t branch_max, int basis = 0) {
    const uint32_t np = p.nparams;
    const uint32_t L = p.n_levels - 1;
    LeafGeom g{};
    g.np = np;
    g.nbins = static_cast<uint32_t>(p.cfg.nbins);
    g.ls = (np + 2) * 2;
    g.n_accel = static_cast<uint32_t>(p.param_counts[L][np - 2]);
    g.n_freq = static_cast<uint32_t>(p.param_counts[L][np - 1]);
    g.eta = p.cfg.eta;
    g.a_min = p.lim_min(np - 2);
    g.a_max = p.lim_max(np - 2);
    g.f_min = p.lim_min(np - 1);
    g.f_max = p.lim_max(np - 1);
    g.branch_max = branch_max;
    g.basis = basis == 1 ? 1u : 0u;
    return g;
}

// poly_chebyshev_transform_*: from (t_cur, s_cur) to (t_next, s_next).
TransformConsts make_transform_cheby(Coord next, Coord cur) {
    TransformConsts tc{};
    tc.basis = 1;
    tc.dt = next.ref - cur.ref;
    tc.p = next.scale / cur.scale;
    tc.q = tc.dt / cur.scale;
    tc.p2 = tc.p * tc.p;
    tc.q2 = tc.q * tc.q;
    tc.pq = tc.p * tc.q;
    tc.p3 = tc.p2 * tc.p;
    return tc;
}

// poly_chebyshev_resolve_*: coordinates add, cur, init.
ResolveConsts make_resolve_cheby(uint32_t np, Coord add, Coord cur, Coord init) {
    ResolveConsts rc{};
    rc.basis = 1;
    const double dt_add = add.ref - cur.ref;
    const double dt_init = init.ref - cur.ref;
    rc.dt_add = dt_add;
    rc.inv_ts = 1.0 / cur.scale;
    rc.inv_ts2 = rc.inv_ts * rc.inv_ts;
    rc.dt = dt_add - dt_init;
    if (np == 2) {
        rc.dt2 = ((dt_add * dt_add) - (dt_init * dt_init));
    } else {
        const double dt2_add = dt_add * dt_add;
        const double dt2_init = dt_init * dt_init;
        rc.dt2 = dt2_add - dt2_init;
        rc.dt3 = (dt2_add * dt_add) - (dt2_init * dt_init);
        rc.inv_ts3 = rc.inv_ts2 * rc.inv_ts;
    }
    return rc;
}

TransformConsts make_transform(uint32_t np, double t_next, double t_cur, bool conservative) {
    TransformConsts tc{};
    tc.dt = t_next - t_cur;
    tc.dt2 = tc.dt * tc.dt;
    tc.half_dt2 = np == 2 ? 0.5 * (tc.dt * tc.dt) : 0.5 * (tc.dt2);
    tc.sixth_dt3 = tc.dt2 * tc.dt / 6.0;
    tc.conservative = conservative ? 1 : 0;
    return tc;
}

ResolveConsts make_resolve(uint32_t np, double t_add, double t_cur, double t_init) {
    ResolveConsts rc{};
    const double dt_add = t_add - t_cur;
    const double dt_init = t_init - t_cur;
    rc.dt_add = dt_add;
    if (np == 2) {
        rc.dt = dt_add - dt_init;
        rc.half_dt2 = 0.5 * ((dt_add * dt_add) - (dt_init * dt_init));
    } else {
        const double half_dt2_add = 0.5 * (dt_add * dt_add);
        const double half_dt2_init = 0.5 * (dt_init * dt_init);
        rc.dt = dt_add - dt_init;
        rc.half_dt2 = half_dt2_add - half_dt2_init;
        rc.sixth_dt3 = ((half_dt2_add * dt_add) - (half_dt2_init * dt_init)) / 3.0;
    }
    return rc;
}

unsigned grid_for(uint64_t n, uint32_t threads) {
    const uint64_t b = (n + threads - 1) / threads;
    require(b <= 0x7fffffffULL, "launch grid too large");
    return static_cast<unsigned>(b < 1 ? 1 : b);
}

// Exclusive scan of n uint32 counts into uint64 offsets, total at d_total.
void scan_counts(const uint32_t* d_x, uint64_t n, uint64_t* d_out, uint32_t* d_sums,
                 uint64_t* d_offs, uint64_t* d_total, cudaStream_t s) {
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    if (n == 0) {
        set_u64_kernel<<<1, 1, 0, s>>>(d_total, 0);
        return;
    }
    scan_tile_sums_kernel<<<grid_for(ntiles, 1), kScanThreads, 0, s>>>(d_x, n, d_sums);
    scan_tiles_kernel<<<1, kScanThreads, 0, s>>>(d_sums, ntiles, d_offs, d_total);
    scan_apply_kernel<<<grid_for(ntiles, 1), kScanThreads, 0, s>>>(d_x, n, d_offs, d_out);
    LK_CUDA(cudaGetLastError());
}

}  // namespace

PruneExec::PruneExec(const Plan& plan, uint64_t max_sugg, uint64_t batch_size,
                     uint64_t branch_max, bool conservative, int device, int basis)
    : m_plan(plan),
      m_device(device),
      m_cap(max_sugg),
      m_batch(batch_size),
      m_branch_max(branch_max),
      m_conservative(conservative),
      m_basis(basis) {
    if (const char* e = std::getenv("LOKI_B200_PRUNE_TAIL")) {
        tail_enabled = std::atoi(e) != 0;
    }
    m_np = plan.nparams;
    require(!plan.offsets_overflow, "coordinate offsets exceed 32 bits");
    require(m_np == 2 || m_np == 3,
            "pruning is implemented for searches with nparams 2 (accel) or 3 (jerk)");
    require(basis == 0 || basis == 1, "poly_basis must be taylor (0) or chebyshev (1)");
    require(!(basis == 1 && conservative),
            "Conservative tile not implemented for Chebyshev basis");
    const uint32_t L = plan.n_levels - 1;
    m_nbins = static_cast<uint32_t>(plan.cfg.nbins);
    m_ls = (m_np + 2) * 2;
    m_nseg = plan.nsegments[L];
    m_tseg = plan.tsegments[L];
    m_ncoords = plan.ncoords[L];
    require(m_nseg >= 1, "pruning needs at least one FFA segment");
    require(m_ncoords == plan.param_counts[L][m_np - 2] * plan.param_counts[L][m_np - 1],
            "n_leaves mismatch: the final FFA level must have one cell in the higher "
            "derivatives");
    require(max_sugg >= 1 && max_sugg < (1ull << 31), "max_sugg must lie in [1, 2^31)");
    require(m_ncoords <= max_sugg, "WorldTree: Suggestions too large to add.");
    require(batch_size >= 1, "batch_size must be positive");
    require(branch_max >= 1, "branch_max must be positive");
    m_sp = make_score_params(plan.widths.data(), static_cast<uint32_t>(plan.widths.size()),
                             m_nbins);
    DeviceGuard g(device);
    for (int i = 0; i < 2; ++i) {
        m_tleaves[i].alloc(m_cap * m_ls * sizeof(double));
        m_tfolds[i].alloc(m_cap * 2 * m_nbins * sizeof(float));
        m_tscores[i].alloc(m_cap * sizeof(float));
        m_lids[i].alloc(m_cap * sizeof(uint32_t));
        m_lsc[i].alloc(m_cap * sizeof(float));
    }
    m_status.alloc(sizeof(uint32_t));
    LK_CUDA(cudaMemset(m_status.ptr, 0, sizeof(uint32_t)));
    m_misc.alloc(kMiscBytes);
    LK_CUDA(cudaMemset(m_misc.ptr, 0, kMiscBytes));
    m_host.alloc(64 * 1024);
}

uint64_t PruneExec::device_bytes() const {
    uint64_t b = m_status.bytes + m_misc.bytes;
    for (int i = 0; i < 2; ++i) {
        b += m_tleaves[i].bytes + m_tfolds[i].bytes + m_tscores[i].bytes + m_lids[i].bytes +
             m_lsc[i].bytes;
    }
    for (const DeviceBuffer* d : {&m_counts, &m_offsets, &m_scan_sums, &m_scan_offs, &m_bparents,
                                  &m_bchild, &m_cleaves, &m_cparent, &m_cscores, &m_cfolds,
                                  &m_bcounts}) {
        b += d->bytes;
    }
    return b;
}

void PruneExec::ensure_level_buffers(uint64_t n_parents, uint64_t n_children) {
    const uint64_t n_scan = std::max({n_parents, n_children, m_cap}) + 1;
    const uint64_t ntiles = (n_scan + kScanTile - 1) / kScanTile + 1;
    if (m_scan_sums.bytes < ntiles * sizeof(uint32_t)) {
        m_scan_sums.alloc(ntiles * sizeof(uint32_t));
        m_scan_offs.alloc(ntiles * sizeof(uint64_t));
    }
    if (n_parents > m_cap_parents) {
        m_counts.alloc(n_parents * sizeof(uint32_t));
        m_offsets.alloc(n_parents * sizeof(uint64_t));
        m_cap_parents = n_parents;
    }
    if (n_children > m_cap_children) {
        m_cleaves.alloc(n_children * m_ls * sizeof(double));
        m_cparent.alloc(n_children * sizeof(uint32_t));
        m_cscores.alloc(n_children * sizeof(float));
        m_cfolds.alloc(n_children * 2 * m_nbins * sizeof(float));
        m_cap_children = n_children;
    }
}

void PruneExec::compact_children(uint64_t c_begin, uint64_t c_end, uint32_t* out_ids,
                                 float* out_sc, const uint64_t* d_base, uint64_t limit,
                                 uint64_t* d_size_out, cudaStream_t s) {
    auto* misc = static_cast<char*>(m_misc.ptr);
    auto* d_thr = reinterpret_cast<const float*>(misc + kMiscThr);
    auto* d_total = reinterpret_cast<uint64_t*>(misc + kMiscTotal);
    const uint64_t n = c_end - c_begin;
    if (n == 0) {
        set_u64_kernel<<<1, 1, 0, s>>>(d_total, 0);
    } else {
        const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
        const auto* sc = m_cscores.as<const float>();
        pc_count_kernel<Src::kChildren, false><<<grid_for(ntiles, 1), kScanThreads, 0, s>>>(
            sc, nullptr, c_begin, n, d_thr, m_scan_sums.as<uint32_t>());
        scan_tiles_kernel<<<1, kScanThreads, 0, s>>>(m_scan_sums.as<uint32_t>(), ntiles,
                                                     m_scan_offs.as<uint64_t>(), d_total);
        pc_scatter_kernel<Src::kChildren, false><<<grid_for(ntiles, 1), kScanThreads, 0, s>>>(
            sc, nullptr, c_begin, n, d_thr, m_scan_offs.as<uint64_t>(), d_base, limit, out_ids,
            out_sc);
    }
    pc_finish_kernel<<<1, 1, 0, s>>>(d_base, d_total, limit, d_size_out);
    LK_CUDA(cudaGetLastError());
}

void PruneExec::compact_list_gt(const uint32_t* ids, const float* sc, uint64_t n,
                                uint32_t* out_ids, float* out_sc, const uint64_t* d_base,
                                uint64_t* d_size_out, cudaStream_t s) {
    auto* misc = static_cast<char*>(m_misc.ptr);
    auto* d_thr = reinterpret_cast<const float*>(misc + kMiscThr);
    auto* d_total = reinterpret_cast<uint64_t*>(misc + kMiscTotal);
    if (n == 0) {
        set_u64_kernel<<<1, 1, 0, s>>>(d_total, 0);
    } else {
        const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
        pc_count_kernel<Src::kList, true><<<grid_for(ntiles, 1), kScanThreads, 0, s>>>(
            sc, ids, 0, n, d_thr, m_scan_sums.as<uint32_t>());
        scan_tiles_kernel<<<1, kScanThreads, 0, s>>>(m_scan_sums.as<uint32_t>(), ntiles,
                                                     m_scan_offs.as<uint64_t>(), d_total);
        pc_scatter_kernel<Src::kList, true><<<grid_for(ntiles, 1), kScanThreads, 0, s>>>(
            sc, ids, 0, n, d_thr, m_scan_offs.as<uint64_t>(), d_base, m_cap, out_ids, out_sc);
    }
    pc_finish_kernel<<<1, 1, 0, s>>>(d_base, d_total, m_cap, d_size_out);
    LK_CUDA(cudaGetLastError());
}

namespace {

__global__ void minmax_kernel(const float* __restrict__ x, uint64_t n, uint32_t* mm) {
    __shared__ uint32_t s_min, s_max;
    if (threadIdx.x == 0) {
        s_min = 0xffffffffu;
        s_max = 0u;
    }
    __syncthreads();
    uint32_t lo = 0xffffffffu, hi = 0u;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t k = fkey(x[i]);
        lo = min(lo, k);
        hi = max(hi, k);
    }
    atomicMin(&s_min, lo);
    atomicMax(&s_max, hi);
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicMin(&mm[0], s_min);
        atomicMax(&mm[1], s_max);
    }
}

}  // namespace

std::vector<lk_prune_stats> PruneExec::run(const float* d_ffa_fold, uint64_t ref_seg,
                                           const float* thresholds, uint64_t n_thresholds,
                                           uint64_t n_iters, cudaStream_t s) {
    PruneRunState rs;
    run_begin(rs, d_ffa_fold, ref_seg, thresholds, n_thresholds, n_iters, s);
    run_levels(rs, false, s);
    return run_end(rs, s);
}

void PruneExec::run_begin(PruneRunState& rs, const float* d_ffa_fold, uint64_t ref_seg,
                          const float* thresholds, uint64_t n_thresholds, uint64_t n_iters,
                          cudaStream_t s) {
    require(d_ffa_fold != nullptr, "ffa_fold is null");
    require(ref_seg < m_nseg, "ref_idx must be less than nsegments.");
    DeviceGuard g(m_device);
    const std::vector<uint64_t> order = middle_out_order(m_nseg, ref_seg);
    const uint64_t seg_floats = m_ncoords * 2 * m_nbins;
    auto* misc = static_cast<char*>(m_misc.ptr);
    auto* d_mm = reinterpret_cast<uint32_t*>(misc + kMiscMinMax);
    LK_CUDA(cudaMemsetAsync(m_status.ptr, 0, sizeof(uint32_t), s));

    // initialize (lib/prune.cpp:181-226): seed leaves, fold segment, scores.
    m_tree = TreeState{};
    m_tree.cap = m_cap;
    m_cur = 0;
    const LeafGeom geom = make_geom(m_plan, m_branch_max, m_basis);
    const uint32_t L = m_plan.n_levels - 1;
    const double dp0 = m_plan.dparams_actual[L][0];
    const double dp1 = m_np == 3 ? m_plan.dparams_actual[L][1] : 0.0;
    const double dfreq = m_plan.dparams_actual[L][m_np - 1];
    seed_kernel<<<grid_for(m_ncoords, 256), 256, 0, s>>>(geom, dp0, dp1, dfreq,
                                                         m_tleaves[0].as<double>());
    if (m_basis == 1) {
        // BaseChebyshevPruneDPFuncts::seed (lib/dynamic.cpp:203-218)
        basis_convert_kernel<<<grid_for(m_ncoords, 256), 256, 0, s>>>(
            m_tleaves[0].as<double>(), m_ncoords, m_np, mo_coord(order, 0, m_tseg).scale, 1);
    }
    const float* seg0 = d_ffa_fold + order[0] * seg_floats;
    LK_CUDA(cudaMemcpyAsync(m_tfolds[0].ptr, seg0, seg_floats * sizeof(float),
                            cudaMemcpyDeviceToDevice, s));
    score_folds(seg0, m_ncoords, m_nbins, true, 1.0f, m_sp, LK_SCORE_MAX,
                m_tscores[0].as<float>(), s);
    init_minmax_kernel<<<1, 1, 0, s>>>(d_mm);
    minmax_kernel<<<std::min<unsigned>(grid_for(m_ncoords, 256), 1184), 256, 0, s>>>(
        m_tscores[0].as<float>(), m_ncoords, d_mm);
    LK_CUDA(cudaGetLastError());
    LK_CUDA(cudaMemcpyAsync(m_host.ptr, d_mm, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    m_tree.size = m_ncoords;
    rs.stats.clear();
    {
        lk_prune_stats s0{};
        s0.level = 0;
        s0.seg_idx = order[0];
        s0.n_branches = s0.n_leaves = s0.n_leaves_phy = s0.n_leaves_surv = m_ncoords;
        s0.threshold = 0.0f;
        s0.score_min = m_ncoords ? key_to_float(m_host.as<uint32_t>()[0]) : 0.0f;
        s0.score_max = m_ncoords ? key_to_float(m_host.as<uint32_t>()[1]) : 0.0f;
        rs.stats.push_back(s0);
    }
    m_order = order;
    m_level = 0;
    m_ran = true;
    m_finalized = false;
    rs.order = order;
    rs.fold = d_ffa_fold;
    rs.thresholds = thresholds;
    rs.n_thresholds = n_thresholds;
    rs.levels = std::min<uint64_t>(m_nseg - 1, n_iters);
    rs.lv = 1;
    rs.handed_back = rs.at_tail = rs.done = false;
    // Each level's score minimum / maximum stays in its own device slot and
    // is read back once, after the last level.
    if (m_level_mm.bytes < 2 * (rs.levels + 1) * sizeof(uint32_t)) {
        m_level_mm.alloc(2 * (rs.levels + 1) * sizeof(uint32_t));
    }
}

void PruneExec::run_levels(PruneRunState& rs, bool stop_at_tail, cudaStream_t s) {
    DeviceGuard g(m_device);
    const uint64_t seg_floats = m_ncoords * 2 * m_nbins;
    rs.at_tail = false;
    // Small trees run in the persistent tail; a level it hands back (too many
    // parents or children) runs here, then the tail is tried again.
    while (!rs.done && rs.lv <= rs.levels) {
        require(rs.lv <= rs.n_thresholds, "Pruning complete - exceeded threshold scheme length");
        if (tail_enabled && !rs.handed_back && m_tree.size <= kTailParents) {
            if (stop_at_tail) {
                rs.at_tail = true;
                return;
            }
            TailArgs a{};
            tail_prepare(rs, &a, s);
            if (m_tail_args.bytes < sizeof(TailArgs)) {
                m_tail_args.alloc(sizeof(TailArgs));
            }
            LK_CUDA(cudaMemcpyAsync(m_tail_args.ptr, &a, sizeof(a), cudaMemcpyHostToDevice, s));
            int dev = 0, nsm = 148;
            LK_CUDA(cudaGetDevice(&dev));
            LK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
            // blocks: one per SM by default (LOKI_B200_PRUNE_TAIL_BLOCKS: fewer)
            if (const char* e = std::getenv("LOKI_B200_PRUNE_TAIL_BLOCKS")) {
                nsm = std::max(1, std::min(nsm, std::atoi(e)));
            }
            launch_tails(m_tail_args.as<TailArgs>(), 1, static_cast<uint32_t>(nsm), m_sp, m_nbins,
                         a.rs, s);
            LK_CUDA(cudaStreamSynchronize(s));
            tail_finish(rs, s);
            continue;
        }
        rs.handed_back = false;
        const float* d_seg = rs.fold + rs.order[rs.lv] * seg_floats;
        lk_prune_stats st{};
        level(d_seg, rs.order, rs.lv, rs.thresholds[rs.lv - 1], &st, s);
        rs.stats.push_back(st);
        m_level = rs.lv;
        ++rs.lv;
        if (m_tree.size == 0) {
            rs.done = true;
        }
    }
    rs.done = true;
}

std::vector<lk_prune_stats> PruneExec::run_end(PruneRunState& rs, cudaStream_t s) {
    DeviceGuard g(m_device);
    std::vector<lk_prune_stats>& stats = rs.stats;
    if (stats.size() > 1) {
        std::vector<uint32_t> mm(2 * stats.size());
        LK_CUDA(cudaMemcpyAsync(mm.data(), m_level_mm.ptr, mm.size() * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, s));
        LK_CUDA(cudaStreamSynchronize(s));
        for (size_t k = 1; k < stats.size(); ++k) {
            const bool any = stats[k].n_leaves > 0;
            stats[k].score_min = any ? key_to_float(mm[2 * k]) : FLT_MAX;
            stats[k].score_max = any ? key_to_float(mm[2 * k + 1]) : -FLT_MAX;
        }
    }
    return std::move(stats);
}

std::vector<std::vector<lk_prune_stats>> PruneExec::run_many(
    const std::vector<PruneExec*>& ex, const float* d_ffa_fold, const std::vector<uint64_t>& ref_segs,
    const float* thresholds, uint64_t n_thresholds, uint64_t n_iters, cudaStream_t s) {
    require(ex.size() == ref_segs.size() && !ex.empty(), "run_many: one executor per reference segment");
    for (size_t k = 1; k < ex.size(); ++k) {
        require(ex[k] != ex[0] && ex[k]->m_device == ex[0]->m_device && ex[k]->m_nbins == ex[0]->m_nbins &&
                    ex[k]->m_sp.nwidths == ex[0]->m_sp.nwidths && ex[k]->m_sp.wmax == ex[0]->m_sp.wmax,
                "run_many: executors of one plan on one device, one per run");
    }
    DeviceGuard g(ex[0]->m_device);
    std::vector<PruneRunState> rs(ex.size());
    // 1. each run up to where its tail would start
    for (size_t k = 0; k < ex.size(); ++k) {
        ex[k]->run_begin(rs[k], d_ffa_fold, ref_segs[k], thresholds, n_thresholds, n_iters, s);
        ex[k]->run_levels(rs[k], true, s);
    }
    // 2. the tails of all runs in one cooperative launch
    std::vector<size_t> at;
    for (size_t k = 0; k < ex.size(); ++k) {
        if (rs[k].at_tail) {
            at.push_back(k);
        }
    }
    if (!at.empty()) {
        std::vector<TailArgs> args(at.size());
        for (size_t i = 0; i < at.size(); ++i) {
            ex[at[i]]->tail_prepare(rs[at[i]], &args[i], s);
        }
        PruneExec* e0 = ex[at[0]];
        if (e0->m_tail_args.bytes < args.size() * sizeof(TailArgs)) {
            e0->m_tail_args.alloc(args.size() * sizeof(TailArgs));
        }
        LK_CUDA(cudaMemcpyAsync(e0->m_tail_args.ptr, args.data(), args.size() * sizeof(TailArgs),
                                cudaMemcpyHostToDevice, s));
        int dev = 0, nsm = 148;
        LK_CUDA(cudaGetDevice(&dev));
        LK_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const uint32_t per_sm = tail_blocks_per_sm(e0->m_sp, e0->m_nbins, args[0].rs);
        const uint32_t total = per_sm * static_cast<uint32_t>(nsm);
        const uint32_t bpt = std::max<uint32_t>(
            1, std::min<uint32_t>(static_cast<uint32_t>(nsm), total / static_cast<uint32_t>(at.size())));
        require(static_cast<uint64_t>(bpt) * at.size() <= total,
                "run_many: more runs than the device holds tail blocks");
        launch_tails(e0->m_tail_args.as<TailArgs>(), static_cast<uint32_t>(at.size()), bpt, e0->m_sp,
                     e0->m_nbins, args[0].rs, s);
        LK_CUDA(cudaStreamSynchronize(s));
        for (size_t i = 0; i < at.size(); ++i) {
            ex[at[i]]->tail_finish(rs[at[i]], s);
        }
    }
    // 3. whatever a tail handed back, and the runs' ends
    std::vector<std::vector<lk_prune_stats>> out(ex.size());
    for (size_t k = 0; k < ex.size(); ++k) {
        ex[k]->run_levels(rs[k], false, s);
        out[k] = ex[k]->run_end(rs[k], s);
    }
    return out;
}

void PruneExec::tail_prepare(PruneRunState& rs, void* args, cudaStream_t s) {
    const uint64_t first = rs.lv;
    const uint64_t last = std::min(rs.levels, rs.n_thresholds);
    const std::vector<uint64_t>& order = rs.order;
    const float* d_ffa_fold = rs.fold;
    const float* thresholds = rs.thresholds;
    const uint64_t seg_floats = m_ncoords * 2 * m_nbins;
    // children buffers: up to kTailChildren, at most 256 MiB of child data
    const uint64_t per_child = m_ls * sizeof(double) + 8 + 2 * m_nbins * sizeof(float);
    const uint64_t max_children = std::min<uint64_t>(kTailChildren, (256ull << 20) / per_child);
    ensure_level_buffers(kTailParents, max_children);
    if (m_tail_tp.bytes < kTailParents * m_ls * sizeof(double)) {
        m_tail_tp.alloc(kTailParents * m_ls * sizeof(double));
    }
    if (m_tail_ctl.bytes < sizeof(TailCtl)) {
        m_tail_ctl.alloc(sizeof(TailCtl));
    }
    if (m_tail_levels.bytes < (last + 1) * sizeof(TailLevel)) {
        m_tail_levels.alloc((last + 1) * sizeof(TailLevel));
    }
    if (m_tail_stats.bytes < 3 * (last + 1) * sizeof(uint64_t)) {
        m_tail_stats.alloc(3 * (last + 1) * sizeof(uint64_t));
    }
    // the level constants, as level() derives them
    std::vector<TailLevel> lc(last + 1);
    const Coord ci = mo_coord(order, 0, m_tseg);
    for (uint64_t lv = first; lv <= last; ++lv) {
        const Coord cp = mo_coord(order, lv - 1, m_tseg);
        const Coord cn = mo_coord(order, lv, m_tseg);
        const Coord cc = mo_current_coord(order, lv, m_tseg);
        const Coord ca = mo_segment_coord(order, lv, m_tseg);
        TailLevel& L = lc[lv];
        L.seg = d_ffa_fold + order[lv] * seg_floats;
        L.threshold = thresholds[lv - 1];
        L.dt = cc.scale;
        L.rc = m_basis == 1 ? make_resolve_cheby(m_np, ca, cc, ci) : make_resolve(m_np, ca.ref, cc.ref, ci.ref);
        L.tc = m_basis == 1 ? make_transform_cheby(cn, cc)
                            : make_transform(m_np, cn.ref, cc.ref, m_conservative);
        L.pt = m_basis == 1 ? make_transform_cheby(cc, cp) : TransformConsts{};
    }
    // pageable sources: the copies are staged before these calls return
    LK_CUDA(cudaMemcpyAsync(m_tail_levels.ptr, lc.data(), lc.size() * sizeof(TailLevel),
                            cudaMemcpyHostToDevice, s));
    TailCtl c{};
    c.head = m_tree.head;
    c.size = m_tree.size;
    c.cur = static_cast<uint32_t>(m_cur);
    c.level = static_cast<uint32_t>(first);
    LK_CUDA(cudaMemcpyAsync(m_tail_ctl.ptr, &c, sizeof(c), cudaMemcpyHostToDevice, s));

    TailArgs& a = *static_cast<TailArgs*>(args);
    a = TailArgs{};
    for (int i = 0; i < 2; ++i) {
        a.tleaves[i] = m_tleaves[i].as<double>();
        a.tfolds[i] = m_tfolds[i].as<float>();
        a.tscores[i] = m_tscores[i].as<float>();
        a.lids[i] = m_lids[i].as<uint32_t>();
        a.lsc[i] = m_lsc[i].as<float>();
    }
    a.cleaves = m_cleaves.as<double>();
    a.cparent = m_cparent.as<uint32_t>();
    a.cscores = m_cscores.as<float>();
    a.cfolds = m_cfolds.as<float>();
    a.tp = m_tail_tp.as<double>();
    a.counts = m_counts.as<uint32_t>();
    a.offsets = m_offsets.as<uint64_t>();
    a.lconst = m_tail_levels.as<TailLevel>();
    a.ctl = m_tail_ctl.as<TailCtl>();
    a.stats = m_tail_stats.as<uint64_t>();
    a.level_mm = m_level_mm.as<uint32_t>();
    a.cap = m_cap;
    a.batch = m_batch;
    a.branch_max = m_branch_max;
    a.max_parents = kTailParents;
    a.max_children = max_children;
    a.last_level = static_cast<uint32_t>(last);
    a.rs = sc::row_stride(m_nbins, m_sp.wmax);
    a.geom = make_geom(m_plan, m_branch_max, m_basis);
    a.sp = m_sp;
}

void PruneExec::tail_finish(PruneRunState& rs, cudaStream_t s) {
    const uint64_t first = rs.lv;
    const uint64_t last = std::min(rs.levels, rs.n_thresholds);
    TailCtl c{};
    std::vector<uint64_t> st(3 * (last + 1));
    LK_CUDA(cudaMemcpyAsync(&c, m_tail_ctl.ptr, sizeof(c), cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaMemcpyAsync(st.data(), m_tail_stats.ptr, st.size() * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    if (c.status & dev::kStatusWaitTimeout) {
        fail(LK_ERR_DEVICE_TIMEOUT, "pruning tail: a grid barrier gave up waiting");
    }
    if (c.exit == kTailExitError) {
        if (c.status & kStatusBranchMax) {
            fail(LK_ERR_INVALID_ARG, "num_points must be less than or equal to branch_max");
        }
        if (c.status & kStatusZeroStep) {
            fail(LK_ERR_INVALID_ARG, "Both dparam_cur and dparam_new must be positive");
        }
        if (c.status & kStatusBranchCount) {
            fail(LK_ERR_UNSUPPORTED, "a parent has more than 2^32-1 children");
        }
        if (c.reason == kTailReasonBatch) {
            fail(LK_ERR_INVALID_ARG,
                 "Branch factor exceeded workspace size:n_leaves_batch <= max_branched_leaves");
        }
        fail(LK_ERR_UNSUPPORTED, "more than 2^32 children in one level");
    }
    for (uint64_t lv = first; lv < c.level; ++lv) {
        lk_prune_stats r{};
        r.level = lv;
        r.seg_idx = rs.order[lv];
        r.n_branches = st[3 * lv];
        r.n_leaves = st[3 * lv + 1];
        r.n_leaves_phy = st[3 * lv + 1];
        r.n_leaves_surv = st[3 * lv + 2];
        r.threshold = rs.thresholds[lv - 1];
        r.score_min = FLT_MAX;   // filled by run_end from the level's device slot
        r.score_max = -FLT_MAX;
        rs.stats.push_back(r);
        m_level = lv;
    }
    m_tree.head = c.head;
    m_tree.size = c.size;
    m_tree.size_old = 0;
    m_tree.read_consumed = 0;
    m_tree.write_start = (c.head + c.size) % m_tree.cap;
    m_cur = static_cast<int>(c.cur);
    rs.lv = c.level;
    rs.at_tail = false;
    // stopped before the last level with leaves left: handed back
    rs.handed_back = m_tree.size > 0 && rs.lv <= last;
    if (m_tree.size == 0) {
        rs.done = true;
    }
}

void PruneExec::level(const float* d_seg, const std::vector<uint64_t>& order, uint64_t lv,
                      float threshold, lk_prune_stats* st, cudaStream_t s) {
    TreeState& t = m_tree;
    auto* misc = static_cast<char*>(m_misc.ptr);
    auto* d_thr = reinterpret_cast<float*>(misc + kMiscThr);
    auto* d_zero = reinterpret_cast<uint64_t*>(misc + kMiscZero);
    uint64_t* d_size[2] = {reinterpret_cast<uint64_t*>(misc + kMiscSize0),
                           reinterpret_cast<uint64_t*>(misc + kMiscSize1)};
    auto* d_total = reinterpret_cast<uint64_t*>(misc + kMiscTotal);
    auto* d_mm = m_level_mm.as<uint32_t>() + 2 * lv;  // this level's min / max keys

    // prepare_in_place_update (lib/world_tree.cpp:237-249)
    t.size_old = t.size;
    t.write_start = (t.head + t.size) % t.cap;
    t.size = 0;
    t.read_consumed = 0;
    const uint64_t n_par = t.size_old;
    const Coord ci = mo_coord(order, 0, m_tseg);
    const Coord cp = mo_coord(order, lv - 1, m_tseg);
    const Coord cn = mo_coord(order, lv, m_tseg);
    const Coord cc = mo_current_coord(order, lv, m_tseg);
    const Coord ca = mo_segment_coord(order, lv, m_tseg);

    // Batches: get_leaves_span splits a batch at the buffer's wrap
    // (lib/world_tree.cpp:148-163, lib/prune.cpp:509-530).
    std::vector<uint64_t> bstart, bsize;
    {
        const uint64_t bs = std::max<uint64_t>(1, std::min(m_batch, n_par));
        uint64_t done = 0;
        while (done < n_par) {
            const uint64_t want = std::min(bs, n_par - done);
            const uint64_t phys = (t.head + done) % t.cap;
            const uint64_t take = std::min(want, t.cap - phys);
            bstart.push_back(done);
            bsize.push_back(take);
            done += take;
        }
    }
    const uint64_t nbat = bstart.size();
    const size_t host_need = 64 + (nbat + 1) * sizeof(uint64_t) * 2 + nbat * sizeof(uint32_t);
    if (m_host.bytes < host_need) {
        LK_CUDA(cudaStreamSynchronize(s));
        m_host.alloc(host_need * 2);
    }
    if (m_cap_batches < nbat + 1) {
        m_bparents.alloc((nbat + 1) * sizeof(uint64_t));
        m_bchild.alloc((nbat + 1) * sizeof(uint64_t));
        m_bcounts.alloc((nbat + 1) * sizeof(uint32_t));
        m_cap_batches = nbat + 1;
    }
    auto* h = static_cast<char*>(m_host.ptr);
    auto* h_bpar = reinterpret_cast<uint64_t*>(h + 64);
    auto* h_bchild = h_bpar + (nbat + 1);
    auto* h_counts = reinterpret_cast<uint32_t*>(h_bchild + (nbat + 1));
    for (uint64_t b = 0; b < nbat; ++b) {
        h_bpar[b] = bstart[b];
    }
    h_bpar[nbat] = n_par;
    ensure_level_buffers(n_par, 0);

    // 1. branch: counts, offsets, batch child ranges. In the Chebyshev basis
    // the parents are first re-centred in place from coord_prev to
    // coord_cur (every batch's branch does this to its parents).
    const LeafGeom geom = make_geom(m_plan, m_branch_max, m_basis);
    if (m_basis == 1 && n_par > 0) {
        parent_transform_kernel<<<grid_for(n_par, 256), 256, 0, s>>>(
            m_tleaves[m_cur].as<double>(), t.head, t.cap, n_par, m_np,
            make_transform_cheby(cc, cp));
    }
    const double* tree_leaves = m_tleaves[m_cur].as<double>();
    // nothing before the batch replay reads the threshold or the list size,
    // and nothing before the leaf kernel the min / max slot
    level_init_kernel<<<1, 1, 0, s>>>(d_thr, threshold, d_size[0], d_mm);
    LK_CUDA(cudaMemcpyAsync(m_bparents.ptr, h_bpar, (nbat + 1) * sizeof(uint64_t),
                            cudaMemcpyHostToDevice, s));
    branch_count_kernel<<<grid_for(n_par, 256), 256, 0, s>>>(
        tree_leaves, t.head, t.cap, n_par, cc.scale, geom, m_counts.as<uint32_t>(),
        m_status.as<uint32_t>());
    scan_counts(m_counts.as<uint32_t>(), n_par, m_offsets.as<uint64_t>(),
                m_scan_sums.as<uint32_t>(), m_scan_offs.as<uint64_t>(), d_total, s);
    batch_child_starts_kernel<<<grid_for(nbat + 1, 256), 256, 0, s>>>(
        m_offsets.as<uint64_t>(), n_par, d_total, m_bparents.as<uint64_t>(), nbat + 1,
        m_bchild.as<uint64_t>());
    LK_CUDA(cudaGetLastError());
    LK_CUDA(cudaMemcpyAsync(h_bchild, m_bchild.ptr, (nbat + 1) * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaMemcpyAsync(h, m_status.ptr, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    const uint32_t status = *reinterpret_cast<uint32_t*>(h);
    if (status & kStatusBranchMax) {
        fail(LK_ERR_INVALID_ARG, "num_points must be less than or equal to branch_max");
    }
    if (status & kStatusZeroStep) {
        fail(LK_ERR_INVALID_ARG, "Both dparam_cur and dparam_new must be positive");
    }
    if (status & kStatusBranchCount) {
        fail(LK_ERR_UNSUPPORTED, "a parent has more than 2^32-1 children");
    }
    const std::vector<uint64_t> cstart(h_bchild, h_bchild + nbat + 1);
    const uint64_t n_child = cstart[nbat];
    for (uint64_t b = 0; b < nbat; ++b) {
        if (cstart[b + 1] - cstart[b] > m_batch * m_branch_max) {
            fail(LK_ERR_INVALID_ARG,
                 "Branch factor exceeded workspace size:n_leaves_batch <= max_branched_leaves");
        }
    }
    require(n_child < (1ull << 32), "more than 2^32 children in one level");
    ensure_level_buffers(n_par, n_child);

    // 2. children: leaves, then resolve + shift-add + score (+ kept folds)
    branch_emit_kernel<<<grid_for(n_par, 256), 256, 0, s>>>(
        tree_leaves, t.head, t.cap, n_par, cc.scale, geom, m_offsets.as<uint64_t>(),
        m_cleaves.as<double>(), m_cparent.as<uint32_t>(), m_status.as<uint32_t>());
    if (n_child > 0) {
        const ResolveConsts rc = m_basis == 1 ? make_resolve_cheby(m_np, ca, cc, ci)
                                              : make_resolve(m_np, ca.ref, cc.ref, ci.ref);
        const uint32_t rs = sc::row_stride(m_nbins, m_sp.wmax);
        const uint32_t T = sc::profiles_per_block(rs + 4);
        const size_t smem = static_cast<size_t>(T) * rs * sizeof(float) + 4 * T * sizeof(uint32_t);
        auto launch = [&](auto kern) {
            sc::set_smem(kern, smem);
            kern<<<grid_for(n_child, T), T, smem, s>>>(
                m_cleaves.as<double>(), m_cparent.as<uint32_t>(), n_child,
                m_tfolds[m_cur].as<float>(), t.head, t.cap, d_seg, geom, rc, rs, m_sp,
                threshold, m_cscores.as<float>(), m_cfolds.as<float>(), d_mm);
        };
        sc::dispatch_nw_nb(m_sp.nwidths, m_nbins, [&](auto nw, auto nbc) {
            launch(leaf_kernel<decltype(nw)::value, decltype(nbc)::value>);
        });
        LK_CUDA(cudaGetLastError());
    }

    // 3. filter + add, batch by batch in the reference's order
    int li = 0;
    uint64_t b = 0;
    bool size_known = true;  // t.size (0 here) matches the device's list size
    while (b < nbat) {
        batch_count_kernel<<<static_cast<unsigned>(nbat - b), 256, 0, s>>>(
            m_cscores.as<float>(), m_bchild.as<uint64_t>(), b, d_thr, m_bcounts.as<uint32_t>());
        LK_CUDA(cudaGetLastError());
        LK_CUDA(cudaMemcpyAsync(h_counts, m_bcounts.ptr, (nbat - b) * sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, s));
        LK_CUDA(cudaMemcpyAsync(h, d_size[li], sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        LK_CUDA(cudaStreamSynchronize(s));
        t.size = *reinterpret_cast<uint64_t*>(h);
        size_known = true;
        // fast path of add_batch_scattered (lib/world_tree.cpp:376-384)
        uint64_t bf = b;
        while (bf < nbat) {
            const uint64_t cnt = h_counts[bf - b];
            if (cnt > t.space_left()) {
                break;
            }
            t.size += cnt;
            t.read_consumed += bsize[bf];
            ++bf;
        }
        if (bf > b) {
            compact_children(cstart[b], cstart[bf], m_lids[li].as<uint32_t>(),
                             m_lsc[li].as<float>(), d_size[li], m_cap, d_size[li], s);
        }
        if (bf == nbat) {
            break;
        }
        // overload (lib/world_tree.cpp:386-421)
        const uint64_t space = t.space_left();
        const uint64_t K = t.size + space;
        const uint64_t N = t.size + h_counts[bf - b];
        const uint64_t m = N / 2;
        const uint64_t r_med = (m <= K - 1) ? (K - 1 - m) : (N - 1 - m + K);
        select_threshold_kernel<<<1, 1024, 0, s>>>(m_lsc[li].as<float>(), t.size,
                                                   m_cscores.as<float>(), cstart[bf],
                                                   cstart[bf + 1], N, K - 1, r_med, d_thr,
                                                   reinterpret_cast<float*>(misc + kMiscDebug));
        LK_CUDA(cudaGetLastError());
        compact_list_gt(m_lids[li].as<uint32_t>(), m_lsc[li].as<float>(), t.size,
                        m_lids[1 - li].as<uint32_t>(), m_lsc[1 - li].as<float>(), d_zero,
                        d_size[1 - li], s);
        compact_children(cstart[bf], cstart[bf + 1], m_lids[1 - li].as<uint32_t>(),
                         m_lsc[1 - li].as<float>(), d_size[1 - li], K, d_size[1 - li], s);
        li = 1 - li;
        t.read_consumed += bsize[bf];
        b = bf + 1;
        size_known = false;  // the overload step's size is on the device
    }
    if (!size_known) {
        LK_CUDA(cudaMemcpyAsync(h, d_size[li], sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        LK_CUDA(cudaStreamSynchronize(s));
        t.size = *reinterpret_cast<uint64_t*>(h);
    }

    // 4. transform + gather into the other tree buffer; finalize_in_place_update
    if (t.size > 0) {
        const TransformConsts tc = m_basis == 1 ? make_transform_cheby(cn, cc)
                                                : make_transform(m_np, cn.ref, cc.ref, m_conservative);
        const int nxt = 1 - m_cur;
        gather_kernel<<<grid_for(t.size * kWarp, 256), 256, 0, s>>>(
            m_lids[li].as<uint32_t>(), m_lsc[li].as<float>(), t.size, m_cleaves.as<double>(),
            m_cfolds.as<float>(), t.write_start, t.cap, m_np, m_nbins, tc,
            m_tleaves[nxt].as<double>(), m_tfolds[nxt].as<float>(), m_tscores[nxt].as<float>());
        LK_CUDA(cudaGetLastError());
        m_cur = nxt;
    }
    t.head = t.write_start;
    t.size_old = 0;
    t.read_consumed = 0;

    st->level = lv;
    st->seg_idx = order[lv];
    st->n_branches = n_par;
    st->n_leaves = n_child;
    st->n_leaves_phy = n_child;
    st->n_leaves_surv = t.size;
    st->threshold = threshold;
    // score_min / score_max: filled by run() from this level's device slot
    st->score_min = FLT_MAX;
    st->score_max = -FLT_MAX;
}

void PruneExec::finalize(const float* d_ffa_fold, cudaStream_t s) {
    require(d_ffa_fold != nullptr, "ffa_fold is null");
    require(m_ran, "finalize needs a pruning run first");
    require(!m_finalized, "the run's survivors are already ascended and reported");
    DeviceGuard g(m_device);
    m_finalized = true;
    const TreeState& t = m_tree;
    if (t.size == 0) {
        return;  // ascend_survivors_batched returns on an empty tree
    }
    const uint64_t nsegs = m_level + 1;
    std::vector<uint32_t> segs(nsegs);
    for (uint64_t k = 0; k < nsegs; ++k) {
        segs[k] = static_cast<uint32_t>(m_order[k]);
    }
    if (m_segs.bytes < m_nseg * sizeof(uint32_t)) {
        m_segs.alloc(m_nseg * sizeof(uint32_t));
    }
    if (m_tscores_ep.bytes < m_cap * sizeof(float)) {
        m_tscores_ep.alloc(m_cap * sizeof(float));
    }
    // the copy reads pageable host memory: it completes before returning
    LK_CUDA(cudaMemcpyAsync(m_segs.ptr, segs.data(), nsegs * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s));
    const Coord mid = mo_coord(m_order, m_level, m_tseg);
    const LeafGeom geom = make_geom(m_plan, m_branch_max, m_basis);
    const uint32_t rs = sc::row_stride(m_nbins, m_sp.wmax);
    // per thread: its scoring row and its share of the warp accumulators
    const uint32_t T = sc::profiles_per_block(rs + (2 * m_nbins + kWarp - 1) / kWarp);
    const size_t smem = (static_cast<size_t>(T) * rs + static_cast<size_t>(T / kWarp) * 2 * m_nbins) *
                        sizeof(float);
    auto launch = [&](auto kern) {
        sc::set_smem(kern, smem);
        kern<<<grid_for(t.size, T), T, smem, s>>>(
            m_tleaves[m_cur].as<double>(), t.head, t.cap, t.size, d_ffa_fold, m_ncoords,
            m_segs.as<uint32_t>(), static_cast<uint32_t>(nsegs), m_tseg, mid.ref, 1.0 / mid.scale,
            geom, rs, m_sp, m_tfolds[m_cur].as<float>(), m_tscores[m_cur].as<float>(),
            m_tscores_ep.as<float>());
    };
    sc::dispatch_nw_nb(m_sp.nwidths, m_nbins, [&](auto nw, auto nbc) {
        launch(ascend_kernel<decltype(nw)::value, decltype(nbc)::value>);
    });
    report_kernel<<<grid_for(t.size, 256), 256, 0, s>>>(m_tleaves[m_cur].as<double>(), t.head,
                                                        t.cap, t.size, m_np,
                                                        static_cast<uint32_t>(m_basis), mid.scale);
    LK_CUDA(cudaGetLastError());
}

void PruneExec::copy_scores_ep(float* d_scores_ep, cudaStream_t s) const {
    require(m_finalized, "scores_ep exist after finalize");
    DeviceGuard g(m_device);
    const TreeState& t = m_tree;
    if (d_scores_ep == nullptr || t.size == 0) {
        return;
    }
    const uint64_t first = std::min(t.size, t.cap - t.head);
    const uint64_t second = t.size - first;
    LK_CUDA(cudaMemcpyAsync(d_scores_ep, m_tscores_ep.as<float>() + t.head, first * sizeof(float),
                            cudaMemcpyDeviceToDevice, s));
    if (second > 0) {
        LK_CUDA(cudaMemcpyAsync(d_scores_ep + first, m_tscores_ep.ptr, second * sizeof(float),
                                cudaMemcpyDeviceToDevice, s));
    }
}

void PruneExec::copy_tree(double* d_leaves, float* d_folds, float* d_scores,
                          cudaStream_t s) const {
    DeviceGuard g(m_device);
    const TreeState& t = m_tree;
    const uint64_t first = std::min(t.size, t.cap - t.head);
    const uint64_t second = t.size - first;
    const size_t lb = m_ls * sizeof(double), fb = 2 * m_nbins * sizeof(float);
    auto cp = [&](void* dst, const DeviceBuffer& src, size_t unit) {
        if (dst == nullptr) {
            return;
        }
        LK_CUDA(cudaMemcpyAsync(dst, static_cast<const char*>(src.ptr) + t.head * unit,
                                first * unit, cudaMemcpyDeviceToDevice, s));
        if (second > 0) {
            LK_CUDA(cudaMemcpyAsync(static_cast<char*>(dst) + first * unit, src.ptr,
                                    second * unit, cudaMemcpyDeviceToDevice, s));
        }
    };
    cp(d_leaves, m_tleaves[m_cur], lb);
    cp(d_folds, m_tfolds[m_cur], fb);
    cp(d_scores, m_tscores[m_cur], sizeof(float));
}

}  // namespace lk

// ---- single steps ----------------------------------------------------------

namespace lk {

namespace {

__global__ void resolve_kernel(const double* __restrict__ leaves, uint64_t n, LeafGeom g,
                               ResolveConsts rc, uint32_t* __restrict__ pidx,
                               float* __restrict__ phase) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) {
        resolve_leaf(leaves + i * g.ls, g, rc, pidx + i, phase + i);
    }
}

// kernels::shift_add_linear_batch (lib/kernels.cpp:1328-1355), warp per leaf.
// The reference wraps (index + start) once; an index that lands outside the
// tree or an FFA row beyond n_ffa is skipped and flagged instead.
__global__ void shift_add_kernel(const float* __restrict__ tree, const uint32_t* __restrict__ it,
                                 const float* __restrict__ ffa, const uint32_t* __restrict__ iff,
                                 const float* __restrict__ phase, float* __restrict__ out,
                                 uint32_t nb, uint64_t n, uint64_t pstart, uint64_t cap,
                                 uint64_t n_ffa, uint32_t* status) {
    const uint64_t w = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp;
    const uint32_t lane = threadIdx.x % kWarp;
    if (w >= n) {
        return;
    }
    const uint64_t logical = static_cast<uint64_t>(it[w]) + pstart;
    const uint64_t phys = logical < cap ? logical : logical - cap;
    const uint64_t row = iff[w];
    if (phys >= cap || row >= n_ffa) {
        if (lane == 0) {
            atomicOr(status, dev::kStatusBadTable);
        }
        return;
    }
    const float* tail = tree + phys * 2 * nb;
    const float* hd = ffa + row * 2 * nb;
    const uint32_t s = dev::shift_bins(phase[w], nb);
    float* o = out + w * 2 * nb;
    for (uint32_t j = lane; j < nb; j += kWarp) {
        const uint32_t jh = j >= s ? j - s : j + nb - s;
        o[j] = __fadd_rn(tail[j], hd[jh]);
        o[nb + j] = __fadd_rn(tail[nb + j], hd[nb + jh]);
    }
}

void require_taylor(const Plan& plan) {
    require(plan.nparams == 2 || plan.nparams == 3,
            "pruning is implemented for searches with nparams 2 (accel) or 3 (jerk)");
}

uint64_t branch_impl(const Plan& plan, const double* d_leaves, uint64_t n, double scale_cur,
                     uint64_t branch_max, double* d_out, uint32_t* d_origins, uint64_t max_out,
                     cudaStream_t s, int basis);

}  // namespace

void taylor_seed(const Plan& plan, double* d_leaves, cudaStream_t s) {
    require_taylor(plan);
    const uint32_t L = plan.n_levels - 1;
    const uint32_t np = plan.nparams;
    require(plan.ncoords[L] == plan.param_counts[L][np - 2] * plan.param_counts[L][np - 1],
            "n_leaves mismatch");
    const LeafGeom g = make_geom(plan, 1);
    const double dp0 = plan.dparams_actual[L][0];
    const double dp1 = np == 3 ? plan.dparams_actual[L][1] : 0.0;
    seed_kernel<<<grid_for(plan.ncoords[L], 256), 256, 0, s>>>(
        g, dp0, dp1, plan.dparams_actual[L][np - 1], d_leaves);
    LK_CUDA(cudaGetLastError());
}

uint64_t taylor_branch(const Plan& plan, const double* d_leaves, uint64_t n, double scale_cur,
                       uint64_t branch_max, double* d_out, uint32_t* d_origins, uint64_t max_out,
                       cudaStream_t s) {
    return branch_impl(plan, d_leaves, n, scale_cur, branch_max, d_out, d_origins, max_out, s, 0);
}

uint64_t cheby_branch(const Plan& plan, double* d_leaves, uint64_t n, double t_cur, double s_cur,
                      double t_prev, double s_prev, uint64_t branch_max, double* d_out,
                      uint32_t* d_origins, uint64_t max_out, cudaStream_t s) {
    require_taylor(plan);
    if (n > 0) {
        parent_transform_kernel<<<grid_for(n, 256), 256, 0, s>>>(
            d_leaves, 0, n, n, plan.nparams,
            make_transform_cheby(Coord{t_cur, s_cur}, Coord{t_prev, s_prev}));
        LK_CUDA(cudaGetLastError());
    }
    return branch_impl(plan, d_leaves, n, 0.0, branch_max, d_out, d_origins, max_out, s, 1);
}

void cheby_resolve(const Plan& plan, const double* d_leaves, uint64_t n, const double* coords,
                   uint32_t* d_param_idx, float* d_phase_shift, cudaStream_t s) {
    require_taylor(plan);
    if (n == 0) {
        return;
    }
    const LeafGeom g = make_geom(plan, 1, 1);
    const ResolveConsts rc = make_resolve_cheby(plan.nparams, Coord{coords[0], coords[1]},
                                                Coord{coords[2], coords[3]},
                                                Coord{coords[4], coords[5]});
    resolve_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_leaves, n, g, rc, d_param_idx,
                                                    d_phase_shift);
    LK_CUDA(cudaGetLastError());
}

void basis_convert(double* d_leaves, uint64_t n, uint32_t nparams, double ts, bool to_cheby,
                   cudaStream_t s) {
    require(nparams == 2 || nparams == 3, "basis conversion supports nparams 2 or 3");
    require(ts > 0.0, "the coordinate scale must be positive");
    if (n == 0) {
        return;
    }
    basis_convert_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_leaves, n, nparams, ts,
                                                          to_cheby ? 1 : 0);
    LK_CUDA(cudaGetLastError());
}

namespace {

uint64_t branch_impl(const Plan& plan, const double* d_leaves, uint64_t n, double scale_cur,
                     uint64_t branch_max, double* d_out, uint32_t* d_origins, uint64_t max_out,
                     cudaStream_t s, int basis) {
    require_taylor(plan);
    require(branch_max >= 1, "branch_max must be positive");
    if (n == 0) {
        return 0;
    }
    const LeafGeom g = make_geom(plan, branch_max, basis);
    DeviceBuffer counts(n * sizeof(uint32_t)), offsets(n * sizeof(uint64_t));
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    DeviceBuffer sums(ntiles * sizeof(uint32_t)), offs(ntiles * sizeof(uint64_t));
    DeviceBuffer misc(16);
    LK_CUDA(cudaMemsetAsync(misc.ptr, 0, 16, s));
    auto* d_status = reinterpret_cast<uint32_t*>(static_cast<char*>(misc.ptr) + 8);
    auto* d_total = misc.as<uint64_t>();
    branch_count_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_leaves, 0, n, n, scale_cur, g,
                                                         counts.as<uint32_t>(), d_status);
    scan_counts(counts.as<uint32_t>(), n, offsets.as<uint64_t>(), sums.as<uint32_t>(),
                offs.as<uint64_t>(), d_total, s);
    uint64_t host[2] = {0, 0};
    LK_CUDA(cudaMemcpyAsync(host, misc.ptr, 16, cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    const uint32_t status = static_cast<uint32_t>(host[1]);
    if (status & kStatusBranchMax) {
        fail(LK_ERR_INVALID_ARG, "num_points must be less than or equal to branch_max");
    }
    if (status & (kStatusZeroStep | kStatusBranchCount)) {
        fail(LK_ERR_INVALID_ARG, "Both dparam_cur and dparam_new must be positive");
    }
    const uint64_t total = host[0];
    if (total <= max_out && total > 0) {
        branch_emit_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_leaves, 0, n, n, scale_cur, g,
                                                            offsets.as<uint64_t>(), d_out,
                                                            d_origins, d_status);
        LK_CUDA(cudaGetLastError());
        LK_CUDA(cudaStreamSynchronize(s));
    }
    return total;
}

}  // namespace

void taylor_resolve(const Plan& plan, const double* d_leaves, uint64_t n, const double* coords,
                    uint32_t* d_param_idx, float* d_phase_shift, cudaStream_t s) {
    require_taylor(plan);
    if (n == 0) {
        return;
    }
    const LeafGeom g = make_geom(plan, 1);
    const ResolveConsts rc = make_resolve(plan.nparams, coords[0], coords[2], coords[4]);
    resolve_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_leaves, n, g, rc, d_param_idx,
                                                    d_phase_shift);
    LK_CUDA(cudaGetLastError());
}

namespace {

// Reads a one-word device status after the stream's work and turns a set
// bad-index bit into an error.
void check_index_status(const DeviceBuffer& st, cudaStream_t s, const char* what) {
    uint32_t v = 0;
    LK_CUDA(cudaMemcpyAsync(&v, st.ptr, sizeof(v), cudaMemcpyDeviceToHost, s));
    LK_CUDA(cudaStreamSynchronize(s));
    if (v & dev::kStatusBadTable) {
        fail(LK_ERR_INVALID_ARG, what);
    }
}

}  // namespace

void taylor_transform(const Plan& plan, double* d_leaves, uint64_t n_leaves,
                      const uint32_t* d_indices, uint64_t n, double t_next, double t_cur,
                      bool conservative, cudaStream_t s) {
    require_taylor(plan);
    if (n == 0) {
        return;
    }
    const TransformConsts tc = make_transform(plan.nparams, t_next, t_cur, conservative);
    DeviceBuffer st(sizeof(uint32_t));
    LK_CUDA(cudaMemsetAsync(st.ptr, 0, sizeof(uint32_t), s));
    transform_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_leaves, n_leaves, d_indices, n,
                                                      plan.nparams, tc, st.as<uint32_t>());
    LK_CUDA(cudaGetLastError());
    check_index_status(st, s, "transform: an index is at or beyond n_leaves");
}

void cheby_transform(const Plan& plan, double* d_leaves, uint64_t n_leaves,
                     const uint32_t* d_indices, uint64_t n, double t_next, double s_next,
                     double t_cur, double s_cur, cudaStream_t s) {
    require_taylor(plan);
    if (n == 0) {
        return;
    }
    const TransformConsts tc = make_transform_cheby(Coord{t_next, s_next}, Coord{t_cur, s_cur});
    DeviceBuffer st(sizeof(uint32_t));
    LK_CUDA(cudaMemsetAsync(st.ptr, 0, sizeof(uint32_t), s));
    transform_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_leaves, n_leaves, d_indices, n,
                                                      plan.nparams, tc, st.as<uint32_t>());
    LK_CUDA(cudaGetLastError());
    check_index_status(st, s, "transform: an index is at or beyond n_leaves");
}

void shift_add_batch(const float* d_folds_tree, const uint32_t* d_indices_tree,
                     const float* d_folds_ffa, uint64_t n_ffa, const uint32_t* d_indices_ffa,
                     const float* d_phase_shift, float* d_out, uint32_t nbins, uint64_t n,
                     uint64_t physical_start, uint64_t capacity, cudaStream_t s) {
    require(nbins >= 1, "nbins must be positive");
    require(capacity >= 1, "capacity must be positive");
    if (n == 0) {
        return;
    }
    DeviceBuffer st(sizeof(uint32_t));
    LK_CUDA(cudaMemsetAsync(st.ptr, 0, sizeof(uint32_t), s));
    shift_add_kernel<<<grid_for(n * kWarp, 256), 256, 0, s>>>(
        d_folds_tree, d_indices_tree, d_folds_ffa, d_indices_ffa, d_phase_shift, d_out, nbins, n,
        physical_start, capacity, n_ffa, st.as<uint32_t>());
    LK_CUDA(cudaGetLastError());
    check_index_status(st, s,
                       "shift_add: a tree index (wrapped once) or an FFA row index is out of range");
}

}  // namespace lk
