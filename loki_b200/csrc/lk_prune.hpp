// Host side of the GPU pruning leaf step (kernels in prune.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "lk_ffa.hpp"
#include "lk_internal.hpp"
#include "lk_kernels.hpp"

namespace lk {

// Pinned host staging for the few values a level reads back.
struct PinnedBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    void alloc(size_t n) {
        release();
        if (n > 0) {
            LK_CUDA(cudaHostAlloc(&ptr, n, cudaHostAllocDefault));
        }
        bytes = n;
    }
    void release() {
        if (ptr != nullptr) {
            cudaFreeHost(ptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
    ~PinnedBuffer() { release(); }
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// The reference's WorldTree bookkeeping (lib/world_tree.cpp:206-276,557-568),
// replayed on the host; the data lives on the device.
struct TreeState {
    uint64_t cap = 0;
    uint64_t head = 0, size = 0, size_old = 0, write_start = 0, read_consumed = 0;
    uint64_t space_left() const { return cap - ((size_old - read_consumed) + size); }
};

// Where a pruning run stands between its steps (see PruneExec::run).
struct PruneRunState {
    std::vector<uint64_t> order;   // middle-out segment order
    const float* fold = nullptr;   // device FFA fold of the last level
    const float* thresholds = nullptr;
    uint64_t n_thresholds = 0;
    uint64_t levels = 0;           // last level to run
    uint64_t lv = 1;               // next level to run
    bool handed_back = false;      // the tail gave level lv back
    bool at_tail = false;          // stopped where the tail would start
    bool done = false;
    std::vector<lk_prune_stats> stats;
};

// One pruning run over the final FFA level of a plan (EPMultiPass's per
// ref_seg PruneImpl, lib/prune.cpp:40-226,429-620).
class PruneExec {
public:
    // basis: 0 Taylor, 1 Chebyshev (PrunePolyChebyshevDPFuncts, lib/dynamic.cpp:381-450).
    PruneExec(const Plan& plan, uint64_t max_sugg, uint64_t batch_size, uint64_t branch_max,
              bool conservative, int device, int basis = 0);
    // Seeds from segment ref_seg of d_ffa_fold ([nsegments, ncoords, 2, nbins])
    // and runs up to n_iters levels with thresholds[level - 1]. Returns one
    // stats row for the seed and one per level run (stops early when no
    // leaf survives). Synchronises `s` a few times per level.
    std::vector<lk_prune_stats> run(const float* d_ffa_fold, uint64_t ref_seg,
                                    const float* thresholds, uint64_t n_thresholds,
                                    uint64_t n_iters, cudaStream_t s);
    // Several runs (one executor each, same plan and sizes) on one stream:
    // each run's large levels level by level, then the small trees' tails of
    // all runs in ONE cooperative launch (its blocks split between the
    // trees), then whatever a tail handed back. Results are each run's.
    static std::vector<std::vector<lk_prune_stats>> run_many(
        const std::vector<PruneExec*>& ex, const float* d_ffa_fold,
        const std::vector<uint64_t>& ref_segs, const float* thresholds, uint64_t n_thresholds,
        uint64_t n_iters, cudaStream_t s);
    // The end of PruneImpl::run (lib/prune.cpp:136-139): the survivors
    // ascended to the middle of the data (folds over every segment searched,
    // scores of those folds; the run's scores kept as scores_ep) and their
    // leaves reported there (observer-frame Taylor parameters). Once per run.
    void finalize(const float* d_ffa_fold, cudaStream_t s);
    void copy_scores_ep(float* d_scores_ep, cudaStream_t s) const;
    bool finalized() const { return m_finalized; }
    uint64_t tree_size() const { return m_tree.size; }
    // Final tree in logical order into caller device buffers.
    void copy_tree(double* d_leaves, float* d_folds, float* d_scores, cudaStream_t s) const;
    uint64_t device_bytes() const;
    const Plan& plan() const { return m_plan; }

private:
    void ensure_level_buffers(uint64_t n_parents, uint64_t n_children);
    void run_begin(PruneRunState& rs, const float* d_ffa_fold, uint64_t ref_seg,
                   const float* thresholds, uint64_t n_thresholds, uint64_t n_iters, cudaStream_t s);
    // Levels from rs.lv on; with stop_at_tail, returns where the tail would
    // start (rs.at_tail) instead of launching it.
    void run_levels(PruneRunState& rs, bool stop_at_tail, cudaStream_t s);
    std::vector<lk_prune_stats> run_end(PruneRunState& rs, cudaStream_t s);
    // The tail (see prune.cu): prepare uploads this run's level constants and
    // state and fills the host TailArgs at args; finish reads the state back
    // (after the launch has been synchronised) and continues rs.
    void tail_prepare(PruneRunState& rs, void* args, cudaStream_t s);
    void tail_finish(PruneRunState& rs, cudaStream_t s);
    void level(const float* d_seg, const std::vector<uint64_t>& order, uint64_t level,
               float threshold, lk_prune_stats* st, cudaStream_t s);
    void compact_children(uint64_t c_begin, uint64_t c_end, uint32_t* out_ids, float* out_sc,
                          const uint64_t* d_base, uint64_t limit, uint64_t* d_size_out,
                          cudaStream_t s);
    void compact_list_gt(const uint32_t* ids, const float* sc, uint64_t n, uint32_t* out_ids,
                         float* out_sc, const uint64_t* d_base, uint64_t* d_size_out,
                         cudaStream_t s);

    Plan m_plan;
    int m_device;
    uint64_t m_cap, m_batch, m_branch_max;
    bool m_conservative;
    int m_basis = 0;
    uint32_t m_np, m_nbins, m_ls;
    uint64_t m_ncoords, m_nseg;
    double m_tseg;
    ScoreParams m_sp{};
    TreeState m_tree;
    int m_cur = 0;                   // tree buffer holding the current tree
    DeviceBuffer m_tleaves[2], m_tfolds[2], m_tscores[2];
    DeviceBuffer m_lids[2], m_lsc[2];  // write-region list (child id, score)
    DeviceBuffer m_status, m_misc;     // misc: thr, sizes, totals, minmax
    // level buffers
    DeviceBuffer m_counts, m_offsets, m_scan_sums, m_scan_offs, m_bparents, m_bchild;
    DeviceBuffer m_cleaves, m_cparent, m_cscores, m_cfolds, m_bcounts;
    uint64_t m_cap_parents = 0, m_cap_children = 0, m_cap_batches = 0;
    PinnedBuffer m_host;
    // the last run, for finalize
    std::vector<uint64_t> m_order;
    uint64_t m_level = 0;
    bool m_ran = false, m_finalized = false;
    DeviceBuffer m_segs, m_tscores_ep;
    DeviceBuffer m_level_mm;  // per level: orderable min / max score keys
public:
    // The persistent tail (on by default; LOKI_B200_PRUNE_TAIL=0 turns it off).
    bool tail_enabled = true;
private:
    DeviceBuffer m_tail_ctl, m_tail_levels, m_tail_stats, m_tail_tp, m_tail_args;
};

// Single steps (the Taylor PruneDPFuncts interface, include/loki/core/
// dynamic.hpp:22-115), for the C ABI's standalone entry points.
void taylor_seed(const Plan& plan, double* d_leaves, cudaStream_t s);
uint64_t taylor_branch(const Plan& plan, const double* d_leaves, uint64_t n, double scale_cur,
                       uint64_t branch_max, double* d_out, uint32_t* d_origins, uint64_t max_out,
                       cudaStream_t s);
void taylor_resolve(const Plan& plan, const double* d_leaves, uint64_t n, const double* coords,
                    uint32_t* d_param_idx, float* d_phase_shift, cudaStream_t s);
void taylor_transform(const Plan& plan, double* d_leaves, uint64_t n_leaves,
                      const uint32_t* d_indices, uint64_t n, double t_next, double t_cur,
                      bool conservative, cudaStream_t s);
// Chebyshev basis (lib/chebyshev.cpp). cheby_branch re-centres d_leaves in
// place (coord_prev -> coord_cur) before branching, as the reference does;
// coords for resolve = {t_add, s_add, t_cur, s_cur, t_init, s_init}.
uint64_t cheby_branch(const Plan& plan, double* d_leaves, uint64_t n, double t_cur, double s_cur,
                      double t_prev, double s_prev, uint64_t branch_max, double* d_out,
                      uint32_t* d_origins, uint64_t max_out, cudaStream_t s);
void cheby_resolve(const Plan& plan, const double* d_leaves, uint64_t n, const double* coords,
                   uint32_t* d_param_idx, float* d_phase_shift, cudaStream_t s);
void cheby_transform(const Plan& plan, double* d_leaves, uint64_t n_leaves,
                     const uint32_t* d_indices, uint64_t n, double t_next, double s_next,
                     double t_cur, double s_cur, cudaStream_t s);
// poly_taylor_to_cheby (to_cheby, ts = coord_init scale) / poly_cheby_to_taylor.
void basis_convert(double* d_leaves, uint64_t n, uint32_t nparams, double ts, bool to_cheby,
                   cudaStream_t s);
void shift_add_batch(const float* d_folds_tree, const uint32_t* d_indices_tree,
                     const float* d_folds_ffa, uint64_t n_ffa, const uint32_t* d_indices_ffa,
                     const float* d_phase_shift, float* d_out, uint32_t nbins, uint64_t n,
                     uint64_t physical_start, uint64_t capacity, cudaStream_t s);

}  // namespace lk
