// Host-side interfaces of the device building blocks (implemented in .cu files).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include "lk_internal.hpp"

namespace lk {

// RAII device allocation.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) { alloc(n); }
    void alloc(size_t n) {
        release();
        if (n > 0) {
            LK_CUDA(cudaMalloc(&ptr, n));
        }
        bytes = n;
    }
    void release() {
        if (ptr != nullptr) {
            cudaFree(ptr);
        }
        ptr = nullptr;
        bytes = 0;
    }
    ~DeviceBuffer() { release(); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

// Brute fold of a time series into [nseg, nfreq, 2, nbins] FP32.
//
// Plan-time tables: for every trial frequency the sample -> phase-bin map of
// one segment (identical for all segments) is encoded as run-start bits per
// 32 samples plus the bin of each run. Replaying the runs in order adds every
// sample to its bin in increasing sample order, which is the reference's
// summation order (lib/kernels.cpp:550-580), so the fold is bit-identical.
class BruteFoldDevice {
public:
    BruteFoldDevice(const std::vector<double>& freqs, uint64_t segment_len, uint64_t nbins,
                    uint64_t nsamps, double tsamp, double t_ref, uint32_t* d_status);
    // Enqueue the fold of (d_ts_e, d_ts_v); d_fold must hold nseg * nfreq * 2 *
    // nbins floats.
    void execute(const float* d_ts_e, const float* d_ts_v, float* d_fold, cudaStream_t s) {
        bind_inputs(d_ts_e, d_ts_v, s);
        fold(d_fold, s);
    }
    // Points the input tensor maps at the series, or at nbatch series of
    // nsamps samples stored back to back. fold() then folds all of them:
    // d_fold holds nbatch * fold_size() floats. With both rows per warp the
    // series are first interleaved into (e, v) pairs on `s` (one kernel);
    // otherwise the maps read them in place (a misaligned series is first
    // copied into an aligned buffer on `s`).
    void bind_inputs(const float* d_ts_e, const float* d_ts_v, cudaStream_t s,
                     uint64_t nbatch = 1);
    // True when bind_inputs launches the interleave kernel.
    bool interleaves() const { return m_rows == 2; }
    // Launch shape (see brute_fold.cu); false when it does not fit. tmem:
    // consumer warps (of `warps`) whose sums live in tensor memory (packed
    // form only).
    bool configure(uint32_t rows, uint32_t warps, uint32_t stages, uint32_t tmem = 0);
    uint32_t max_warps(uint32_t rows, uint32_t stages) const;
    // Most tensor-memory warps a block of smem_warps shared-memory warps can add.
    uint32_t max_tmem_warps(uint32_t smem_warps) const;
    uint32_t rows() const { return m_rows; }
    uint32_t warps() const { return m_warps; }
    uint32_t stages() const { return m_stages; }
    uint32_t tmem_warps() const { return m_tmem; }
    // d_lens (device, one uint64 per bound series, or nullptr): samples of
    // each series that may be nonzero (the rest must be zero). With both rows
    // per warp and nseg a multiple of 8, only the segments holding them are
    // folded (in groups of 8) and the others' folds are set to +0.0, the
    // result folding the zeros gives; otherwise every segment is folded.
    void fold(float* d_fold, cudaStream_t s, const uint64_t* d_lens = nullptr);
    uint64_t nseg() const { return m_nseg; }
    uint64_t nfreq() const { return m_nfreq; }
    uint64_t fold_size() const { return m_nseg * m_nfreq * 2 * m_nbins; }
    uint64_t device_bytes() const;

private:
    uint64_t m_nfreq, m_seglen, m_nbins, m_nsamps, m_nseg = 0;
    uint64_t m_nwords = 0;
    bool m_wide_bins = false;  // uint16 run bins (nbins > 256)
    uint32_t m_rows = 2;       // rows (E, V) per consumer warp
    uint32_t m_warps = 0;      // consumer warps per block
    uint32_t m_stages = 0;     // shared-memory ring depth (32-sample words)
    uint32_t m_tmem = 0;       // consumer warps with tensor-memory sums
    size_t m_smem = 0;         // dynamic shared memory per block
    uint32_t* m_status;
    DeviceBuffer m_masks;      // uint32 [nfreq][ceil(seglen / 32)] run-start bits
    DeviceBuffer m_bins;       // run bins, all frequencies
    DeviceBuffer m_bin_off;    // uint64 first run of each frequency
    DeviceBuffer m_nruns;      // uint64 runs of each frequency
    DeviceBuffer m_seq;        // uint8 per frequency: run bins step by one
    uint64_t m_nseq = 0;
    DeviceBuffer m_stage;      // aligned copy of a misaligned series
    DeviceBuffer m_ev;         // (e, v) interleaved series (both rows per warp)
    CUtensorMap m_tmap_e{}, m_tmap_v{};
    CUtensorMap m_tmap_ev{};
    CUtensorMap m_tmap_ev8{};  // same rows, 8-row boxes (group mode)
    DeviceBuffer m_groups;     // uint32 group table of the bound batch (group mode)
    const void* m_map_ev_ptr = nullptr;
    const float* m_map_e_ptr = nullptr;
    const float* m_map_v_ptr = nullptr;
    uint64_t m_map_batch = 1;
};

// One merge level: out[s, c] = rot(in[2s, tail(c)], st(c)) + rot(in[2s+1, head(c)], sh(c)).
// Coordinates are [n_outer][n_inner] (n_inner = frequency cells).
// Storage of input / output: FP32, or BF16 when the flag is set (adds are FP32).
void merge_level(const void* d_in, void* d_out, const void* d_coords, bool taylor,
                 uint64_t n_inner, uint64_t n_outer, uint64_t ncoords_prev, uint64_t nsegments,
                 uint32_t nbins, cudaStream_t s, bool in_bf16 = false, bool out_bf16 = false,
                 int pb = 0);

// Boxcar scoring parameters shared by the score kernels.
struct ScoreParams {
    uint32_t nwidths;
    uint32_t wmax;
    uint32_t widths[LK_MAX_WIDTHS];
    float hb[LK_MAX_WIDTHS];  // h + b
    float b[LK_MAX_WIDTHS];
};
ScoreParams make_score_params(const uint32_t* widths, uint32_t nwidths, uint32_t nbins);

// ---- final level for 32 / 64 / 128 bins (final_level.cu) -----------------
// 1 / sqrt(n) table for exact integer variance sums n < kNormTableSize
// (rcp_rn(sqrt_rn(n)), the direct computation's bits).
constexpr uint32_t kNormTableSize = 1u << 19;
void norm_table_fill(float* d_tab, cudaStream_t s);
// Scoring widths as a bit mask (bit w for width w <= 32) with the per-width
// constants and output slots, for strictly increasing widths.
struct MaskScoreParams {
    uint64_t wmask;
    uint32_t nwidths;
    uint32_t wmax;
    float hb[33];
    float b[33];
    uint8_t slot[33];
};
// False when the masked path does not apply (nbins not 32 / 64 / 128, widths
// not strictly increasing or wider than 32 bins).
bool make_mask_score_params(const ScoreParams& sp, uint32_t nbins, MaskScoreParams* mp);
uint32_t final_level_cells_per_block();
// Blocks (count slots) of one final-level launch.
uint64_t final_level_blocks(uint64_t n_inner, uint64_t n_outer, uint64_t nbatch);
// Final merge level fused with scoring (same results as merge_score_level).
// With d_counts, each block also writes its number of scores >= count_thr
// (per-width mode) to d_counts[final_level_blocks order].
void merge_score_level_wm(const void* d_in, const void* d_coords, bool taylor, uint64_t n_inner,
                          uint64_t n_outer, uint64_t ncoords_prev, uint32_t nbins,
                          const MaskScoreParams& mp, int mode, float* d_scores, cudaStream_t s,
                          uint64_t nbatch, bool in_bf16, float* d_cmax, const float* d_tab,
                          float count_thr, uint32_t* d_counts, bool use_table = true);
// Ordered compaction of scores >= thr from the block counts of
// merge_score_level_wm: exclusive scan of the counts (d_offsets: one uint64
// per block), then a scatter of the blocks that have candidates.
void compact_ranges(const float* d_scores, const uint32_t* d_counts, uint64_t* d_offsets,
                    uint64_t n_inner, uint64_t n_outer, uint64_t nbatch, uint32_t nw, float thr,
                    uint32_t* d_idx, float* d_vals, uint64_t max_out, uint64_t* d_count,
                    cudaStream_t s);
// Exclusive scan of n uint32 counts into uint64 offsets (one block); *d_total = sum.
void scan_counts(const uint32_t* d_counts, uint64_t n, uint64_t* d_offsets, uint64_t* d_total,
                 cudaStream_t s);

// Final merge level fused with scoring (one output segment per series;
// nbatch series, the input holding 2 * nbatch segments of ncoords_prev cells,
// scores [nbatch][ncoords][nout]).
void merge_score_level(const void* d_in, const void* d_coords, bool taylor, uint64_t n_inner,
                       uint64_t n_outer, uint64_t ncoords_prev, uint32_t nbins,
                       const ScoreParams& sp, int mode, float* d_scores, cudaStream_t s,
                       uint64_t nbatch = 1, bool in_bf16 = false, float* d_cmax = nullptr,
                       uint32_t cells_per_block = 0);

// Merge tree of the final FFA level: what the exact rescorer needs to rebuild
// one final cell from the FP32 level-0 fold.
constexpr uint32_t kRescoreMaxLevels = 24;
constexpr uint64_t kRescoreMaxLeaves = 8192;  // level-0 segments (2^(levels-1))
struct RescoreTree {
    uint32_t n_levels = 0;
    uint32_t nbins = 0;
    uint64_t ncoords0 = 0;       // rows per level-0 segment
    uint64_t ncoords_final = 0;  // final cells per series
    uint64_t fold0_size = 0;     // floats of one series' level-0 fold
    const void* level_coords[kRescoreMaxLevels] = {};  // device table of level l (l >= 1)
};

// For each of the *d_count final cells listed in d_cells (flat series *
// ncoords_final + coord, at most max_cells of them), rebuilds the FP32 fold
// of that cell from d_fold0 with the merge kernels' exact add tree and writes
// its per-width S/N to d_scores[cell * nwidths ...]: bit-identical to the
// all-FP32 path.
void rescore_cells(const float* d_fold0, const RescoreTree& t, bool taylor, const ScoreParams& sp,
                   const uint32_t* d_cells, const uint64_t* d_count, uint64_t max_cells,
                   float* d_scores, cudaStream_t s);

// Standalone scoring of [nprof, 2, nbins] (is3d) or [nprof, nbins] folds.
void score_folds(const float* d_folds, uint64_t nprof, uint32_t nbins, bool is3d,
                 float inv_stdnoise, const ScoreParams& sp, int mode, float* d_scores,
                 cudaStream_t s);

// cuTensorMapEncodeTiled, resolved from the driver once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// Ordered compaction of scores >= thr.
uint64_t compact_scratch_bytes(uint64_t n);
void compact_ge(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx, float* d_vals,
                uint64_t max_out, uint64_t* d_count, void* d_scratch, cudaStream_t s);
// Same compaction with its scratch in a static device array (n <= 2^28).
// Bounded-wait check: one warp waits (limit_ns) on an mbarrier that is
// completed or never completed; returns the status word (synchronises s).
uint32_t wait_check(uint64_t limit_ns, bool complete, uint32_t* d_status, cudaStream_t s);

void compact_ge_noalloc(const float* d_scores, uint64_t n, float thr, uint32_t* d_idx,
                        float* d_vals, uint64_t max_out, uint64_t* d_count, cudaStream_t s);

}  // namespace lk
