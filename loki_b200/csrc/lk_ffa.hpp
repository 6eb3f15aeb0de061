// FFA executor (internal).
#pragma once

#include <memory>

#include "lk_kernels.hpp"

namespace lk {

// Makes `device` current for the scope, restoring the previous device.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int device) {
        LK_CUDA(cudaGetDevice(&prev));
        if (prev != device) {
            LK_CUDA(cudaSetDevice(device));
        }
        target = device;
    }
    ~DeviceGuard() {
        if (prev >= 0 && prev != target) {
            cudaSetDevice(prev);
        }
    }
    int target = 0;
};

// Optional per-stage CUDA-event timing of one executor call.
struct StageProfiler {
    struct Stage {
        int kind;
        int level;
        uint32_t launches;
        uint64_t bytes;
        cudaEvent_t start;
        cudaEvent_t stop;
    };
    bool enabled = false;
    std::vector<Stage> stages;  // events are reused across calls
    size_t used = 0;
    void reset() { used = 0; }
    // Records the start event of a new stage on `s` (no-op when disabled).
    void begin(int kind, int level, uint32_t launches, uint64_t bytes, cudaStream_t s);
    void end(cudaStream_t s);
    ~StageProfiler();
};

struct FFAExec {
    Plan plan;
    int device;
    StageProfiler prof;
    DeviceBuffer status;   // uint32 device status word
    DeviceBuffer coords;   // all levels, reference layout
    std::unique_ptr<BruteFoldDevice> bf;
    // Intermediate levels. FP32 storage: ping-pong buffers for every level
    // before the last. BF16 storage: level 0 stays FP32 in fold0 (the exact
    // rescorer rebuilds final cells from it) and levels 1 .. L-2 alternate
    // between the two BF16 buffers.
    DeviceBuffer buf[2];
    DeviceBuffer fold0;
    DeviceBuffer scores_tmp;
    DeviceBuffer compact_scratch;
    // BF16 search: per-cell best approximate S/N, the cells to rescore.
    DeviceBuffer cmax, cells, cell_vals, cell_count, cell_scratch;
    ScoreParams sp{};
    // Final level for 32 / 64 / 128 bins and strictly increasing widths <= 32
    // (final_level.cu): width mask, 1 / sqrt(n) table, per-block candidate
    // counts and their offsets (FP32 search).
    bool wm = false;
    MaskScoreParams mp{};
    DeviceBuffer normtab, blk_counts, blk_offsets;
    // The masked final level runs unless a tuning picked the generic kernel
    // (score_cells >= 32: cells per block of the generic kernel); score_cells
    // 1 selects the masked kernel without the 1 / sqrt table.
    bool use_wm() const { return wm && score_cells < 32; }
    bool mixed = false;  // BF16 storage of levels 1 .. L-2
    // A BF16 search rescores every final cell whose approximate best S/N is
    // at least (snr_min - margin_abs) / (1 + margin_rel).
    float margin_abs = 0.0f;
    float margin_rel = 0.0f;
    RescoreTree rtree{};

    uint64_t max_batch = 1;  // series per call (buffers are sized for it)
    // Device array of the valid samples of each series of a batch (or
    // nullptr): the brute fold skips the segments past them (see
    // BruteFoldDevice::fold). Read by every launch, so a captured graph picks
    // up new lengths written into the same array.
    const uint64_t* batch_lens = nullptr;
    // Tuned launch shapes (0: defaults); see autotune.
    int merge_pb = 0;            // merge: output rows per warp in flight
    uint32_t score_cells = 0;    // final level + score: cells per block
    lk_tuning tuning{};          // last autotune result / applied shapes

    // Times launch-shape candidates of the brute fold (rows per warp,
    // consumer warps per block, ring depth), the merges (rows in flight per
    // warp) and the fused final level (cells per block) on the given series,
    // stage by stage, and keeps the fastest of each. Every candidate computes
    // the same sums in the same order, so results do not change.
    lk_tuning autotune(const float* ts_e, const float* ts_v, uint32_t reps, cudaStream_t s);
    void apply_tuning(const lk_tuning& t);

    FFAExec(const Plan& p, int device, int storage, uint64_t max_batch = 1);
    uint64_t device_bytes() const;
    const void* level_coords(uint32_t l) const;
    uint64_t coord_bytes(uint32_t l) const;
    std::vector<lk_stage_time> profile(cudaStream_t s);
    // Lowest approximate best S/N that a BF16 search rescores for snr_min.
    float rescore_threshold(float snr_min) const;
    // All entry points take nbatch series of nsamps samples stored back to
    // back; outputs are the single-series outputs of each, back to back.
    // run_levels runs levels 0 .. last (inclusive) and returns the buffer
    // holding `last` (BF16 when *last_bf16 is set).
    const void* run_levels(const float* ts_e, const float* ts_v, uint32_t last, float* final_out,
                           cudaStream_t s, uint64_t nbatch, bool* last_bf16);
    // With d_counts (masked final level only), per-block counts of scores >=
    // count_thr are written too.
    void scores_impl(const float* ts_e, const float* ts_v, float* d_scores, float* d_cmax,
                     cudaStream_t s, uint64_t nbatch, float count_thr = 0.0f,
                     uint32_t* d_counts = nullptr);
    void execute(const float* ts_e, const float* ts_v, float* fold, uint64_t fold_len,
                 cudaStream_t s, uint64_t nbatch = 1);
    void scores(const float* ts_e, const float* ts_v, float* d_scores, uint64_t len,
                cudaStream_t s, uint64_t nbatch = 1);
    void search(const float* ts_e, const float* ts_v, float snr_min, uint32_t* d_idx,
                float* d_snr, uint64_t max_cands, uint64_t* d_count, cudaStream_t s,
                uint64_t nbatch = 1);
    uint32_t read_status(cudaStream_t s);
    // Cells the last BF16 search rescored (synchronises s).
    uint64_t rescored_cells(cudaStream_t s);
};

}  // namespace lk
