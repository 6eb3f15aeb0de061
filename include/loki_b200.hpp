/* C++20 drop-in classes over the C ABI of loki_b200.h.
 *
 * Mirrors the reference's C++ interface for the time-domain FFA path, so a
 * caller that used loki::search::PulsarSearchConfig and
 * loki::algorithms::FFACUDA<float> switches by changing the namespace:
 *   - PulsarSearchConfig   include/loki/search/configs.hpp:22-164 (the fields
 *                          the FFA path reads; copyable)
 *   - FFAPlan<float>       include/loki/common/plans.hpp (geometry getters)
 *   - FFACUDA<float>       include/loki/algorithms/ffa.hpp:100-153 (PIMPL,
 *                          move-only; host-span, device-span and stream
 *                          overloads of execute)
 *   - FFACUDA<ComplexTypeCUDA>  the Fourier-domain FFA (same header): complex
 *                          folds, plus the overloads that return to time
 *   - compute_ffa_scores_cuda, the reference's convenience function
 *     (lib/ffa_cuda.cu:671-692), through the Fourier path when the config's
 *     use_fourier is set (the reference default), else the time domain.
 * Errors: a failed call throws std::invalid_argument for rejected arguments
 * (the reference throws invalid_argument from its checks) and
 * std::runtime_error otherwise (its DetailedException / CudaException are
 * runtime_errors). Device spans are std::span over device memory.
 */
#ifndef LOKI_B200_HPP
#define LOKI_B200_HPP

#include <cuda/std/complex>
#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <memory>
#include <optional>
#include <span>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "loki_b200.h"

namespace loki_b200 {

using SizeType = std::size_t;
using ComplexType = std::complex<float>;                 // host fold type
using ComplexTypeCUDA = cuda::std::complex<float>;       // device fold type
static_assert(sizeof(ComplexType) == 8 && sizeof(ComplexTypeCUDA) == 8, "interleaved (re, im) floats");

struct ParamLimit {
    double min;
    double max;
};

namespace detail {
inline void check(int rc) {
    if (rc == LK_OK) {
        return;
    }
    const std::string msg = lk_last_error();
    if (rc == LK_ERR_INVALID_ARG) {
        throw std::invalid_argument(msg);
    }
    throw std::runtime_error(msg);
}
inline void check_cuda(cudaError_t e) {
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(e));
    }
}
// Device buffer owned by a host-span call.
template <class T> struct DeviceArray {
    T* ptr = nullptr;
    explicit DeviceArray(SizeType n) { check_cuda(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T))); }
    ~DeviceArray() { cudaFree(ptr); }
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
};
}  // namespace detail

namespace search {

class PulsarSearchConfig {
public:
    PulsarSearchConfig(SizeType nsamps, double tsamp, SizeType nbins, double eta,
                       std::span<const ParamLimit> param_limits, double ducy_max = 0.2,
                       double wtsp = 1.5, bool use_fourier = true, int nthreads = 1,
                       std::optional<SizeType> bseg_brute = std::nullopt,
                       std::optional<SizeType> bseg_ffa = std::nullopt, double snr_min = 5.0,
                       std::span<const SizeType> score_widths = {},
                       SizeType nbins_min_lossy_bf = 64)
        : m_use_fourier(use_fourier), m_nthreads(nthreads), m_nbins_min_lossy_bf(nbins_min_lossy_bf) {
        if (param_limits.empty() || param_limits.size() > LK_MAX_PARAMS) {
            throw std::invalid_argument("param_limits must hold 1 to 5 (min, max) pairs");
        }
        if (score_widths.size() > LK_MAX_WIDTHS) {
            throw std::invalid_argument("at most 32 score widths");
        }
        m_c = lk_config{};
        m_c.nsamps = nsamps;
        m_c.tsamp = tsamp;
        m_c.nbins = nbins;
        m_c.eta = eta;
        m_c.nparams = static_cast<uint32_t>(param_limits.size());
        for (SizeType i = 0; i < param_limits.size(); ++i) {
            m_c.param_limits[2 * i] = param_limits[i].min;
            m_c.param_limits[2 * i + 1] = param_limits[i].max;
        }
        m_c.ducy_max = ducy_max;
        m_c.wtsp = wtsp;
        m_c.bseg_brute = bseg_brute.value_or(0);
        m_c.bseg_ffa = bseg_ffa.value_or(0);
        m_c.snr_min = snr_min;
        m_c.n_score_widths = static_cast<uint32_t>(score_widths.size());
        for (SizeType i = 0; i < score_widths.size(); ++i) {
            m_c.score_widths[i] = static_cast<uint32_t>(score_widths[i]);
        }
        // validate now, as the reference's constructor does
        lk_plan* p = nullptr;
        detail::check(lk_plan_create(&m_c, &p));
        lk_plan_destroy(p);
    }
    SizeType get_nsamps() const noexcept { return m_c.nsamps; }
    double get_tsamp() const noexcept { return m_c.tsamp; }
    SizeType get_nbins() const noexcept { return m_c.nbins; }
    double get_eta() const noexcept { return m_c.eta; }
    SizeType get_nparams() const noexcept { return m_c.nparams; }
    double get_ducy_max() const noexcept { return m_c.ducy_max; }
    double get_wtsp() const noexcept { return m_c.wtsp; }
    bool get_use_fourier() const noexcept { return m_use_fourier; }
    int get_nthreads() const noexcept { return m_nthreads; }
    double get_tobs() const noexcept { return static_cast<double>(m_c.nsamps) * m_c.tsamp; }
    double get_snr_min() const noexcept { return m_c.snr_min; }
    SizeType get_nbins_f() const noexcept { return m_c.nbins / 2 + 1; }
    SizeType get_nbins_min_lossy_bf() const noexcept { return m_nbins_min_lossy_bf; }
    const lk_config& c_config() const noexcept { return m_c; }

private:
    lk_config m_c{};
    bool m_use_fourier;
    int m_nthreads;
    SizeType m_nbins_min_lossy_bf;
};

}  // namespace search

namespace plans {

// FFAPlan<float> and FFAPlan<ComplexType>: the same levels; the complex
// plan's fold sizes count nbins / 2 + 1 harmonics per row and its *_time
// sizes are those of the fold back in time.
template <class FoldType> class FFAPlan {
    static constexpr bool kComplex = !std::is_same_v<FoldType, float>;
    SizeType to_fold(SizeType time_size) const noexcept {
        return kComplex ? time_size / m_info.nbins * (m_info.nbins / 2 + 1) : time_size;
    }

public:
    explicit FFAPlan(const search::PulsarSearchConfig& cfg) {
        lk_plan* p = nullptr;
        detail::check(lk_plan_create(&cfg.c_config(), &p));
        m_plan.reset(p);
        detail::check(lk_plan_get_info(p, &m_info));
    }
    SizeType get_n_levels() const noexcept { return m_info.n_levels; }
    SizeType get_fold_size() const noexcept { return to_fold(m_info.fold_size); }
    SizeType get_buffer_size() const noexcept { return to_fold(m_info.buffer_size); }
    SizeType get_brute_fold_size() const noexcept { return to_fold(m_info.brute_fold_size); }
    SizeType get_fold_size_time() const noexcept { return m_info.fold_size; }
    SizeType get_buffer_size_time() const noexcept {
        return kComplex ? 2 * get_buffer_size() : m_info.buffer_size;
    }
    std::vector<SizeType> get_ncoords() const {
        return {m_info.ncoords, m_info.ncoords + m_info.n_levels};
    }
    std::vector<SizeType> get_segment_lens() const {
        return {m_info.segment_lens, m_info.segment_lens + m_info.n_levels};
    }
    std::vector<SizeType> get_score_widths() const {
        return {m_info.widths, m_info.widths + m_info.n_widths};
    }
    SizeType get_ncoords_final() const noexcept { return m_info.ncoords[m_info.n_levels - 1]; }
    const lk_plan* handle() const noexcept { return m_plan.get(); }

private:
    struct Del {
        void operator()(lk_plan* p) const noexcept { lk_plan_destroy(p); }
    };
    std::unique_ptr<lk_plan, Del> m_plan;
    lk_plan_info m_info{};
};

}  // namespace plans

namespace algorithms {

template <class FoldTypeCUDA> class FFACUDA;

// FFACUDA<float> (include/loki/algorithms/ffa.hpp:100-153): the time-domain
// FFA executor; fold storage FP32 (LK_BF16 stores intermediate levels in BF16).
template <> class FFACUDA<float> {
public:
    explicit FFACUDA(const search::PulsarSearchConfig& cfg, int device_id = 0,
                     int storage = LK_FP32)
        : m_impl(std::make_unique<Impl>(cfg, device_id, storage)) {}
    ~FFACUDA() = default;
    FFACUDA(FFACUDA&&) noexcept = default;
    FFACUDA& operator=(FFACUDA&&) noexcept = default;
    FFACUDA(const FFACUDA&) = delete;
    FFACUDA& operator=(const FFACUDA&) = delete;

    const plans::FFAPlan<float>& get_plan() const noexcept { return m_impl->plan; }

    // Host series in, host fold out (copies inside, on the default stream).
    void execute(std::span<const float> ts_e, std::span<const float> ts_v, std::span<float> fold) {
        const SizeType n = ts_e.size();
        if (ts_v.size() != n) {
            throw std::invalid_argument("ts_e and ts_v must have the same size");
        }
        detail::DeviceArray<float> e(n), v(n), f(fold.size());
        detail::check_cuda(cudaMemcpy(e.ptr, ts_e.data(), n * sizeof(float), cudaMemcpyHostToDevice));
        detail::check_cuda(cudaMemcpy(v.ptr, ts_v.data(), n * sizeof(float), cudaMemcpyHostToDevice));
        execute(std::span<const float>(e.ptr, n), std::span<const float>(v.ptr, n),
                std::span<float>(f.ptr, fold.size()), nullptr);
        detail::check_cuda(cudaMemcpy(fold.data(), f.ptr, fold.size() * sizeof(float), cudaMemcpyDeviceToHost));
    }
    // Device spans, enqueued on `stream` (no synchronisation).
    void execute(std::span<const float> ts_e_d, std::span<const float> ts_v_d, std::span<float> fold_d,
                 cudaStream_t stream) {
        detail::check(lk_ffa_execute(m_impl->ffa.get(), ts_e_d.data(), ts_v_d.data(), fold_d.data(),
                                     fold_d.size(), reinterpret_cast<lk_stream_t>(stream)));
    }
    // compute_ffa_scores on device spans: [ncoords_final][n_widths] S/N.
    void scores(std::span<const float> ts_e_d, std::span<const float> ts_v_d, std::span<float> scores_d,
                cudaStream_t stream) {
        detail::check(lk_ffa_scores(m_impl->ffa.get(), ts_e_d.data(), ts_v_d.data(), scores_d.data(),
                                    scores_d.size(), reinterpret_cast<lk_stream_t>(stream)));
    }

private:
    struct Impl {
        plans::FFAPlan<float> plan;
        struct Del {
            void operator()(lk_ffa* f) const noexcept { lk_ffa_destroy(f); }
        };
        std::unique_ptr<lk_ffa, Del> ffa;
        Impl(const search::PulsarSearchConfig& cfg, int device_id, int storage) : plan(cfg) {
            lk_ffa* f = nullptr;
            detail::check(lk_ffa_create(plan.handle(), device_id, storage, &f));
            ffa.reset(f);
        }
    };
    std::unique_ptr<Impl> m_impl;
};

// FFACUDA<ComplexTypeCUDA>: the Fourier-domain FFA (folds of nbins / 2 + 1
// complex harmonics, fractional-shift phase rotations, inverse real
// transform back to time).
template <> class FFACUDA<ComplexTypeCUDA> {
public:
    explicit FFACUDA(const search::PulsarSearchConfig& cfg, int device_id = 0)
        : m_impl(std::make_unique<Impl>(cfg, device_id)) {}
    ~FFACUDA() = default;
    FFACUDA(FFACUDA&&) noexcept = default;
    FFACUDA& operator=(FFACUDA&&) noexcept = default;
    FFACUDA(const FFACUDA&) = delete;
    FFACUDA& operator=(const FFACUDA&) = delete;

    const plans::FFAPlan<ComplexType>& get_plan() const noexcept { return m_impl->plan; }

    // Host series in, final complex fold out (fold holds >= fold_size values).
    void execute(std::span<const float> ts_e, std::span<const float> ts_v, std::span<ComplexType> fold) {
        const SizeType n = check_inputs(ts_e, ts_v);
        detail::DeviceArray<float> e(n), v(n), f(2 * fold.size());
        copy_in(e, v, ts_e, ts_v);
        execute(std::span<const float>(e.ptr, n), std::span<const float>(v.ptr, n),
                std::span<ComplexTypeCUDA>(reinterpret_cast<ComplexTypeCUDA*>(f.ptr), fold.size()), nullptr);
        detail::check_cuda(cudaMemcpy(fold.data(), f.ptr, fold.size() * sizeof(ComplexType), cudaMemcpyDeviceToHost));
    }
    // Host series in, final fold back in time out (fold holds >= fold_size_time floats;
    // the reference sizes it 2 * buffer_size).
    void execute(std::span<const float> ts_e, std::span<const float> ts_v, std::span<float> fold) {
        const SizeType n = check_inputs(ts_e, ts_v);
        detail::DeviceArray<float> e(n), v(n), f(fold.size());
        copy_in(e, v, ts_e, ts_v);
        execute(std::span<const float>(e.ptr, n), std::span<const float>(v.ptr, n),
                std::span<float>(f.ptr, fold.size()), nullptr);
        detail::check_cuda(cudaMemcpy(fold.data(), f.ptr, fold.size() * sizeof(float), cudaMemcpyDeviceToHost));
    }
    // Device spans, enqueued on `stream`.
    void execute(std::span<const float> ts_e_d, std::span<const float> ts_v_d, std::span<ComplexTypeCUDA> fold_d,
                 cudaStream_t stream) {
        detail::check(lk_fourier_execute(m_impl->ffa.get(), ts_e_d.data(), ts_v_d.data(),
                                         reinterpret_cast<float*>(fold_d.data()), fold_d.size(),
                                         reinterpret_cast<lk_stream_t>(stream)));
    }
    void execute(std::span<const float> ts_e_d, std::span<const float> ts_v_d, std::span<float> fold_d,
                 cudaStream_t stream) {
        detail::check(lk_fourier_execute_time(m_impl->ffa.get(), ts_e_d.data(), ts_v_d.data(), fold_d.data(),
                                              fold_d.size(), reinterpret_cast<lk_stream_t>(stream)));
    }
    // compute_ffa_scores (use_fourier) on device spans: [ncoords_final][n_widths] S/N.
    void scores(std::span<const float> ts_e_d, std::span<const float> ts_v_d, std::span<float> scores_d,
                cudaStream_t stream) {
        detail::check(lk_fourier_scores(m_impl->ffa.get(), ts_e_d.data(), ts_v_d.data(), scores_d.data(),
                                        scores_d.size(), reinterpret_cast<lk_stream_t>(stream)));
    }

private:
    static SizeType check_inputs(std::span<const float> ts_e, std::span<const float> ts_v) {
        if (ts_v.size() != ts_e.size()) {
            throw std::invalid_argument("ts_e and ts_v must have the same size");
        }
        return ts_e.size();
    }
    static void copy_in(detail::DeviceArray<float>& e, detail::DeviceArray<float>& v, std::span<const float> ts_e,
                        std::span<const float> ts_v) {
        detail::check_cuda(cudaMemcpy(e.ptr, ts_e.data(), ts_e.size() * sizeof(float), cudaMemcpyHostToDevice));
        detail::check_cuda(cudaMemcpy(v.ptr, ts_v.data(), ts_v.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    struct Impl {
        plans::FFAPlan<ComplexType> plan;
        struct Del {
            void operator()(lk_fourier* f) const noexcept { lk_fourier_destroy(f); }
        };
        std::unique_ptr<lk_fourier, Del> ffa;
        Impl(const search::PulsarSearchConfig& cfg, int device_id) : plan(cfg) {
            lk_fourier* f = nullptr;
            detail::check(lk_fourier_create(plan.handle(), device_id, cfg.get_nbins_min_lossy_bf(), &f));
            ffa.reset(f);
        }
    };
    std::unique_ptr<Impl> m_impl;
};

// compute_ffa_scores_cuda (the reference's convenience function): host
// series in, host scores [ncoords_final * n_widths] and the time-domain plan
// out; through the Fourier-domain FFA when cfg.get_use_fourier().
inline std::tuple<std::vector<float>, plans::FFAPlan<float>> compute_ffa_scores_cuda(
    std::span<const float> ts_e, std::span<const float> ts_v, const search::PulsarSearchConfig& cfg,
    int device_id = 0) {
    plans::FFAPlan<float> plan(cfg);
    const SizeType n = ts_e.size();
    const SizeType ns = plan.get_ncoords_final() * plan.get_score_widths().size();
    detail::DeviceArray<float> e(n), v(n), s(ns);
    detail::check_cuda(cudaMemcpy(e.ptr, ts_e.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    detail::check_cuda(cudaMemcpy(v.ptr, ts_v.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    const std::span<const float> de(e.ptr, n), dv(v.ptr, n);
    if (cfg.get_use_fourier()) {
        FFACUDA<ComplexTypeCUDA> ffa(cfg, device_id);
        ffa.scores(de, dv, std::span<float>(s.ptr, ns), nullptr);
    } else {
        FFACUDA<float> ffa(cfg, device_id);
        ffa.scores(de, dv, std::span<float>(s.ptr, ns), nullptr);
    }
    std::vector<float> out(ns);
    detail::check_cuda(cudaMemcpy(out.data(), s.ptr, ns * sizeof(float), cudaMemcpyDeviceToHost));
    return {std::move(out), std::move(plan)};
}

}  // namespace algorithms

}  // namespace loki_b200

#endif  // LOKI_B200_HPP
