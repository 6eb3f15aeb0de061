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
    DeviceBuffer buf[2];   // ping-pong intermediate levels
    DeviceBuffer scores_tmp;
    DeviceBuffer compact_scratch;
    ScoreParams sp{};
    bool in_search = false;

    uint64_t max_batch = 1;  // series per call (buffers are sized for it)

    FFAExec(const Plan& p, int device, int storage, uint64_t max_batch = 1);
    uint64_t device_bytes() const;
    const void* level_coords(uint32_t l) const;
    uint64_t coord_bytes(uint32_t l) const;
    std::vector<lk_stage_time> profile(cudaStream_t s);
    // All entry points take nbatch series of nsamps samples stored back to
    // back; outputs are the single-series outputs of each, back to back.
    float* run_levels(const float* ts_e, const float* ts_v, uint32_t last, float* final_out,
                      cudaStream_t s, uint64_t nbatch = 1);
    void execute(const float* ts_e, const float* ts_v, float* fold, uint64_t fold_len,
                 cudaStream_t s, uint64_t nbatch = 1);
    void scores(const float* ts_e, const float* ts_v, float* d_scores, uint64_t len,
                cudaStream_t s, uint64_t nbatch = 1);
    void search(const float* ts_e, const float* ts_v, float snr_min, uint32_t* d_idx,
                float* d_snr, uint64_t max_cands, uint64_t* d_count, cudaStream_t s,
                uint64_t nbatch = 1);
    uint32_t read_status(cudaStream_t s);
};

}  // namespace lk
